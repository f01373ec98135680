"""CPU-side checks of the C ABI library: it loads, exports every entry point
declared in include/abm_capi.h, its host-only routines (JKR radius table,
synthetic-state generator) agree with the oracle and the reference's
invariants, and without a GPU it fails loudly instead of falling back."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

import abm_b200
from abm_b200 import workloads
import oracle_ref as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "abm_capi.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(abm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    names = header_functions()
    assert len(names) >= 20
    lib = ctypes.CDLL(abm_b200.LIB_PATH)
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(abm_b200.EXPORTED) == names


def test_no_gpu_means_error_not_fallback():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    # the failed abm_create hands back a context holding the reason, which the wrapper
    # reads and then releases
    with pytest.raises(RuntimeError, match="ABM_ERR_CUDA.*no CUDA device"):
        abm_b200.Simulation(cap_cells=16)


def test_product_jkr_table_matches_oracle_and_invariants():
    R, Rcell, E0, gamma = 0.8, 0.5, 3900.0, 100.0
    d, r = abm_b200.jkr_radius_table(R, Rcell, E0, gamma, 100)
    do, ro = orc.jkr_table(R, Rcell, E0, gamma, 100)
    assert np.array_equal(d, do)
    np.testing.assert_allclose(r, ro, rtol=1e-14, atol=0)
    Req = R / 2
    for delta, a in zip(d, r):
        rec = a * a / Req - 2 * math.sqrt(math.pi * gamma * a / E0)
        assert abs(rec - delta) <= 1e-13 * max(1.0, a * a / Req)
    # gamma = 0: a = sqrt(Req delta)  (testJKR.cpp:26-49)
    for delta in d:
        assert abs(abm_b200.jkr_contact_radius(delta, Req, E0, 0.0) - math.sqrt(Req * delta)) <= 1e-8


def test_generator_is_seeded_and_core_free():
    a, ia = workloads.biofilm_3d(n=3000, seed=5, disk_radius=52.0, p_contact=0.9)
    b, ib = workloads.biofilm_3d(n=3000, seed=5, disk_radius=52.0, p_contact=0.9)
    c, _ = workloads.biofilm_3d(n=3000, seed=6, disk_radius=52.0, p_contact=0.9)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert workloads.count_close_pairs(a, ia["min_gap"]) == 0
    assert np.all(a[:, 6] >= 0) and np.allclose(np.linalg.norm(a[:, 4:7], axis=1), 1)
    assert np.all((a[:, 13] >= 2) & (a[:, 13] <= 5)) and np.all(a[:, 3] >= 0.8)
    assert ia["mean_contacts_per_cell"] > 1.5


def test_oracle_loop_matches_reference_order_of_operations():
    # iteration counter, clock and rebuild cadence of simulation.hpp:1617-1864
    cells, _ = workloads.biofilm_3d(n=300, seed=4, disk_radius=300 * math.sqrt(300 / 1e5), p_contact=0.9)
    _, p = abm_b200.make_params(iter_update_neighbors=4)
    o = orc.Oracle(p, jkr=orc.jkr_table(0.8, 0.5, 3900.0, 100.0))
    o.set_cells(cells)
    o.loop_init()
    o.iterate(9)
    t, dt, it = o.clock()
    assert it == 9 and dt == p["max_stepsize"]
    s = o.stats()
    assert s["rebuilds"] == 1 + 9 // 4
    assert s["attempts"] == 2 * 9          # trial + unconditional final re-run per iteration


def test_product_variable_gamma_table_matches_oracle():
    d, g, r = abm_b200.jkr_radius_table_variable(0.8, 0.5, 3900.0, 120.0, 100, 60)
    do, go, ro = orc.jkr_table_variable(0.8, 0.5, 3900.0, 120.0, 100, 60)
    assert np.array_equal(d, do) and np.array_equal(g, go)
    np.testing.assert_allclose(r, ro, rtol=1e-13, atol=0)
    # its gamma = 0 column is the Hertz radius sqrt(Req delta), its last the fixed table at 120
    np.testing.assert_allclose(r[:, 0], np.sqrt(0.4 * d), rtol=1e-12, atol=0)
    _, rf = abm_b200.jkr_radius_table(0.8, 0.5, 3900.0, 120.0, 100)
    np.testing.assert_allclose(r[:, -1], rf, rtol=1e-15, atol=0)
