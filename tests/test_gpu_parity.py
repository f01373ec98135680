"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bars (stated here and in the design notes):
  * neighbor pair set and the table's (d, s, t): bit for bit (both sides use
    correctly rounded arithmetic without FMA for the segment distance);
  * forces, velocities, RK states and error norms: normwise relative error
    max|gpu - oracle| / max|oracle| <= 1e-10 per column (FP64 path).
"""
import json
import os

import numpy as np
import pytest

import abm_b200
from abm_b200 import workloads
import oracle_ref as orc

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 1e-10
JKR = orc.jkr_table(0.8, 0.5, 3900.0, 100.0, 100)


def colwise_relerr(a, b):
    """max over columns of max|a - b| / max|b| (0 where the column of b is zero)."""
    a, b = np.asarray(a), np.asarray(b)
    scale = np.abs(b).max(axis=0)
    diff = np.abs(a - b).max(axis=0)
    return float(np.max(np.where(scale > 0, diff / np.where(scale > 0, scale, 1), diff)))


def make_pair(cells, **kw):
    kw.setdefault("cap_cells", max(len(cells), 1) + 16)
    sim = abm_b200.Simulation(jkr_table=JKR, **kw)
    sim.upload_cells(cells)
    o = orc.Oracle(sim.pdict, jkr=JKR)
    o.set_cells(cells)
    return sim, o


def patch_state(n, seed, p_contact=0.9):
    # same density as the 100k / 300 um benchmark disk
    radius = 300.0 * np.sqrt(n / 100000.0)
    cells, _ = workloads.biofilm_3d(n=n, seed=seed, disk_radius=radius, p_contact=p_contact)
    return cells


def parallel_bundle(n_side=8, spacing=1.3, jitter=0.0, seed=0):
    """Cells on a lattice, all along x (exercises the near-parallel branch)."""
    rng = np.random.default_rng(seed)
    rows = []
    for a in range(n_side):
        for b in range(n_side):
            for c in range(2):
                n = np.array([1.0, 0.0, 0.0]) + jitter * rng.normal(size=3)
                n /= np.linalg.norm(n)
                if n[2] < 0:
                    n = -n
                rows.append(([c * 4.2 + 0.3 * (a % 2), a * spacing, 0.8 + b * spacing], n))
    cells = np.zeros((len(rows), 22), order="F")
    for k, (r, n) in enumerate(rows):
        cells[k, 0] = k
        cells[k, 1:4] = r
        cells[k, 4:7] = n
        cells[k, 13], cells[k, 14] = 3.0, 1.5
        cells[k, 17], cells[k, 18], cells[k, 19], cells[k, 20], cells[k, 21] = 100, 720, 100, 1, 100
    return cells


# ---------------------------------------------------------------------------
# segment distance: the reference's known-answer cases and the oracle, bit for bit
# ---------------------------------------------------------------------------
def test_gpu_distance_golden_cases():
    with open(os.path.join(GOLDEN, "dist3d_cases.json")) as f:
        cases = json.load(f)["dist_cases"]
    for c in cases:
        # cell 1 of the case is row index 1 so the table's d runs from it to cell 2
        cells = workloads.two_cell_3d(c["r2"], c["n2"], c["r1"], c["n1"])
        cells[0, 13], cells[0, 14] = 2 * c["half_l2"], c["half_l2"]
        cells[1, 13], cells[1, 14] = 2 * c["half_l1"], c["half_l1"]
        sim, o = make_pair(cells, neighbor_threshold=100.0, Ldiv=20.0)
        assert sim.get_cell_neighbors() == 1
        row = sim.neighbors()[0]
        assert row[0] == 1 and row[1] == 0
        np.testing.assert_allclose(row[2:5], c["d"], atol=1e-8, rtol=0)
        assert abs(row[5] - c["s"]) <= 1e-8 and abs(row[6] - c["t"]) <= 1e-8
        o.build_neighbors()
        assert np.array_equal(sim.neighbors(), o.neighbors())


# ---------------------------------------------------------------------------
# neighbor set (getCellNeighbors): identical rows, bit for bit
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("state", ["patch1", "patch2", "patch_uniform", "bundle", "bundle_jitter"])
def test_gpu_neighbor_table_bitexact(state):
    cells = {"patch1": lambda: patch_state(3000, 1), "patch2": lambda: patch_state(5000, 2),
             "patch_uniform": lambda: patch_state(3000, 3, p_contact=0.0),
             "bundle": lambda: parallel_bundle(), "bundle_jitter": lambda: parallel_bundle(jitter=0.004)}[state]()
    sim, o = make_pair(cells)
    m = sim.get_cell_neighbors()
    mo = o.build_neighbors()
    assert m == mo and m > 0
    g, r = sim.neighbors(), o.neighbors()
    assert np.array_equal(g, r)


def test_gpu_neighbor_edge_sizes():
    for n in (1, 2, 3, 64):
        cells = patch_state(max(n, 2), 7)[:n]
        sim, o = make_pair(cells)
        m = sim.get_cell_neighbors()
        assert m == o.build_neighbors()
        assert np.array_equal(sim.neighbors(), o.neighbors())


def test_gpu_neighbor_overflow_is_reported():
    cells = parallel_bundle(n_side=8, spacing=1.2)
    sim = abm_b200.Simulation(jkr_table=JKR, cap_cells=len(cells), cap_neighbors_per_cell=4)
    sim.upload_cells(cells)
    with pytest.raises(RuntimeError, match="ABM_ERR_CAPACITY"):
        sim.get_cell_neighbors()


# ---------------------------------------------------------------------------
# forces, velocities, one RK attempt
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("adhesion", [1, 0])
def test_gpu_cell_cell_forces(adhesion):
    cells = patch_state(4000, 11)
    sim, o = make_pair(cells, adhesion_mode=adhesion)
    sim.get_cell_neighbors()
    o.build_neighbors()
    err = colwise_relerr(sim.cell_cell_forces(), o.cell_cell_forces())
    assert err <= RTOL, err


def test_gpu_velocities():
    cells = patch_state(4000, 12)
    sim, o = make_pair(cells)
    sim.get_cell_neighbors()
    o.build_neighbors()
    err = colwise_relerr(sim.get_velocities(), o.get_velocities())
    assert err <= RTOL, err


@pytest.mark.parametrize("mode", [1, 2, 3, 4])
def test_gpu_rk_attempt(mode):
    cells = patch_state(3000, 13)
    sim, o = make_pair(cells, integration_mode=mode)
    sim.get_cell_neighbors()
    o.build_neighbors()
    for dt in (1e-6, 1e-4):
        cg, eg, mg = sim.step_runge_kutta_adaptive(dt)
        co, eo, mo = o.rk_attempt(dt)
        assert colwise_relerr(cg, co) <= RTOL
        # the error estimate dt (sum b k - sum b* k) cancels to rounding level, so it is
        # compared against the scale of the step increment dt * v of each column
        inc = dt * np.abs(co[:, 7:13]).max(axis=0)
        assert np.all(np.abs(eg - eo).max(axis=0) <= RTOL * inc)
        y0 = cells[:, 1:7]
        e_scale = (inc / (1e-8 * (1 + np.abs(y0)))).max()
        assert abs(mg - mo) <= RTOL * e_scale


def test_gpu_rk_attempt_with_noise():
    cells = patch_state(2000, 14)
    kw = dict(max_rxy_noise=50.0, max_rz_noise=20.0, max_nxy_noise=5.0, max_nz_noise=2.0)
    sim, o = make_pair(cells, **kw)
    sim.get_cell_neighbors()
    o.build_neighbors()
    cg, eg, mg = sim.step_runge_kutta_adaptive(1e-5, attempt=3)
    co, eo, mo = o.rk_attempt(1e-5, 0, 3)
    assert colwise_relerr(cg, co) <= RTOL


# ---------------------------------------------------------------------------
# the loop body (divide-free): controller, growth, rebuild cadence
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("graphs", [1, 0])
def test_gpu_iterations_match_oracle(graphs):
    cells = patch_state(2000, 21)
    sim, o = make_pair(cells, use_graphs=graphs, iter_update_neighbors=10, max_stepsize=1e-4)
    sim.get_cell_neighbors()
    o.loop_init()
    for _ in range(3):
        s = sim.iterate(12)
        o.iterate(12)
        t, dt, it = sim.clock()
        to, dto, ito = o.clock()
        assert it == ito
        assert abs(t - to) <= 1e-10 * to and abs(dt - dto) <= 1e-10 * dto
        assert colwise_relerr(sim.download_cells(), o.cells()) <= 1e-9
        assert s["attempts"] == o.stats()["attempts"]
        assert np.array_equal(sim.neighbors()[:, :2], o.neighbors()[:, :2])


def test_gpu_iterations_with_growth_no_division():
    cells = patch_state(1500, 22)
    cells[:, 16] = 0.5                      # growth rate; lengths stay below Ldiv
    cells[:, 13] = np.minimum(cells[:, 13], 4.0)
    cells[:, 14] = cells[:, 13] / 2
    sim, o = make_pair(cells, iter_update_neighbors=5, max_stepsize=1e-4)
    sim.get_cell_neighbors()
    o.loop_init()
    sim.iterate(20)
    o.iterate(20)
    assert colwise_relerr(sim.download_cells(), o.cells()) <= 1e-9


# ---------------------------------------------------------------------------
# full size (100k cells): pair set bit for bit, forces normwise
# ---------------------------------------------------------------------------
def test_gpu_full_size_neighbor_set_and_forces():
    cells, _ = workloads.biofilm_3d(n=100000, seed=1, p_contact=0.9)
    sim, o = make_pair(cells)
    m = sim.get_cell_neighbors()
    assert m == o.build_neighbors()
    g = sim.neighbors()
    assert np.array_equal(g, o.neighbors())
    err = colwise_relerr(sim.cell_cell_forces(), o.cell_cell_forces())
    assert err <= RTOL, err
    cg, eg, mg = sim.step_runge_kutta_adaptive(1e-6)
    co, eo, mo = o.rk_attempt(1e-6)
    assert colwise_relerr(cg, co) <= RTOL
    # Newton's third law: translational pair forces sum to zero
    f = sim.cell_cell_forces()
    assert np.abs(f[:, :3].sum(0)).max() <= 1e-9 * np.abs(f[:, :3]).sum()


# ---------------------------------------------------------------------------
# division (growth.hpp:66-426): who divides, append order, IDs, lineage, the
# number of tries and the daughters' state bit for bit (the draws use
# correctly rounded operations only, on both sides)
# ---------------------------------------------------------------------------
DIV_KW = dict(growth_mean=1.5, growth_std=0.1, daughter_length_std=0.05, daughter_angle_xy_bound=0.3,
              daughter_angle_z_bound=0.1, rng_seed=7)


def dividing_state(n=600, seed=31, n_long=40, crowd=True):
    cells = patch_state(n, seed)
    rng = np.random.default_rng(seed)
    idx = rng.choice(n, n_long, replace=False)
    cells[idx, 13] = 5.7
    cells[idx, 14] = 5.7 / 2
    cells[:, 16] = rng.normal(1.5, 0.1, size=n)
    if crowd:
        # squeeze a few mothers next to a neighbor so they have no room to rotate
        for k in idx[:5]:
            j = (k + 1) % n
            cells[j, 1:4] = cells[k, 1:4] + np.array([0.0, 0.0, 0.95])
            cells[j, 4:7] = cells[k, 4:7]
    return cells, idx


def test_gpu_division_matches_oracle():
    cells, idx = dividing_state()
    n = len(cells)
    sim, o = make_pair(cells, cap_cells=2 * n, **DIV_KW)
    parents = -np.ones(n, dtype=np.int32)
    sim.set_parents(parents)
    o.set_parents(parents)
    sim.set_clock(0.25, 1e-6, 17)
    o.set_clock(0.25, 1e-6, 17)
    nd = sim.divide_cells()
    tries_o = o.divide(0.25, 17)
    assert nd == len(idx) == int((cells[:, 13] > 5.6).sum())
    assert sim.last_division_tries() == tries_o
    cg, co = sim.download_cells(), o.cells()
    assert cg.shape == co.shape == (n + nd, 22)
    assert np.array_equal(cg[:, 0], co[:, 0])                   # IDs
    assert np.array_equal(sim.parents(), o.parents())           # lineage
    assert np.array_equal(cg, co)                               # daughters bit for bit


@pytest.mark.parametrize("graphs", [1, 0])
def test_gpu_growth_and_division_loop(graphs):
    # Per-step parity from identical inputs: each iteration starts both sides from the
    # oracle's state (cells, neighbor table, clock, lineage).  Free-running trajectories
    # are not compared here: two daughters of one mother start exactly 2R apart, where
    # the JKR force jumps at zero overlap (adhesion.hpp:282-370), so a one-ulp
    # difference in an earlier step decides whether the siblings touch.
    cells = patch_state(400, 33)
    rng = np.random.default_rng(3)
    cells[:, 13] = rng.uniform(4.5, 5.55, size=len(cells))
    cells[:40, 13] = 5.6 - rng.uniform(0.0, 2e-3, size=40)      # about to cross Ldiv
    cells[:, 14] = cells[:, 13] / 2
    cells[:, 16] = rng.normal(1.5, 0.1, size=len(cells))
    n = len(cells)
    sim, o = make_pair(cells, cap_cells=3 * n, use_graphs=graphs, max_stepsize=1e-3, iter_update_neighbors=7,
                       **DIV_KW)
    parents = -np.ones(n, dtype=np.int32)
    o.set_parents(parents)
    o.loop_init()
    divided = 0
    for it in range(24):
        sim.upload_cells(o.cells())
        sim.set_neighbors(o.neighbors())
        sim.set_clock(*o.clock())
        sim.set_parents(o.parents())
        n0 = o.cells().shape[0]
        s = sim.iterate(1)
        o.iterate(1)
        cg, co = sim.download_cells(), o.cells()
        assert cg.shape == co.shape
        divided += co.shape[0] - n0
        assert np.array_equal(cg[:, 0], co[:, 0])                # IDs
        assert np.array_equal(sim.parents(), o.parents())        # lineage
        assert colwise_relerr(cg, co) <= 1e-9
        t, dt, i = sim.clock()
        to, dto, io = o.clock()
        assert i == io and abs(dt - dto) <= 1e-10 * dto
        if i % 7 == 0 or co.shape[0] != n0:                      # a rebuild happened
            assert np.array_equal(sim.neighbors()[:, :2], o.neighbors()[:, :2])
    assert divided > 0


@pytest.mark.parametrize("controller", [0, 1])
def test_gpu_iterations_per_graph_change_nothing(controller):
    # abm_iterate launches iter_k iterations per graph when it can (here 10, the largest of
    # 10, 5, 4, 2 dividing iter_update_neighbors); the same 35 iterations launched one at a
    # time must end bit for bit in the same state, divisions and rebuilds included
    from abm_b200 import stepsize
    cells = patch_state(400, 35)
    rng = np.random.default_rng(5)
    cells[:, 13] = rng.uniform(4.5, 5.55, size=len(cells))
    cells[:30, 13] = 5.6 - rng.uniform(0.0, 2e-3, size=30)
    cells[:, 14] = cells[:, 13] / 2
    cells[:, 16] = rng.normal(1.5, 0.1, size=len(cells))
    out = []
    for per_call in (35, 1):
        sim = abm_b200.Simulation(jkr_table=JKR, cap_cells=3 * len(cells), max_stepsize=1e-3,
                                  iter_update_neighbors=10, controller=controller, **DIV_KW)
        sim.upload_cells(cells)
        if controller:
            sim.set_stepsize_weights(stepsize.load())
        sim.set_parents(-np.ones(len(cells), dtype=np.int32))
        sim.set_clock(0.0, 1e-4, 0)
        sim.get_cell_neighbors()
        for _ in range(35 // per_call):
            s = sim.iterate(per_call)
        out.append((sim.download_cells(), sim.parents(), sim.clock(), s))
        sim.close()
    (ca, pa, ta, sa), (cb, pb, tb, sb) = out
    assert sa["divisions"] > 0 and sa["rebuilds"] > 3
    assert np.array_equal(ca, cb) and np.array_equal(pa, pb) and ta == tb
    for k in ("iterations", "attempts", "retries", "rejected", "divisions", "rebuilds"):
        assert sa[k] == sb[k], k
