"""abm_cell_cell_forces_noalloc: the cell-cell force entry point for callers that
cannot allocate device memory (their memory belongs to another allocator, or
they cannot take cudaMalloc's synchronisation in a step loop).  It must give the
same dE/dq as abm_cell_cell_forces and as the CPU oracle on buffers the caller
already owns, call after call, with its scratch in the library's fixed device
array; a neighbor CSR that fails the device-side check must never be used to
index memory, and the failure must reach the caller.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import abm_b200
from abm_b200 import workloads
import oracle_ref as orc

pytestmark = pytest.mark.gpu

JKR = orc.jkr_table(0.8, 0.5, 3900.0, 100.0, 100)
MAX_CELLS, MAX_ENTRIES = 32768, 524288
# FP64 bar of the parity tests; the FP32 pair force loses up to ~1e-5 relative in the
# overlap 2R - |d| of nearly touching cells (cancellation against |d| ~ 2R), so the
# mixed path is held to 1e-4 normwise per column
RTOL_FP64, RTOL_MIXED = 1e-10, 1e-4


def state(n, seed):
    cells, _ = workloads.biofilm_3d(n=n, seed=seed, disk_radius=300.0 * (n / 1e5) ** 0.5, p_contact=0.9)
    return cells


def csr_from_pairs(i, j, n):
    """Both directions of each unordered pair (i, j), every row sorted ascending."""
    i = np.asarray(i, dtype=np.int64)
    j = np.asarray(j, dtype=np.int64)
    src = np.concatenate([i, j])
    dst = np.concatenate([j, i])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(row_ptr, src + 1, 1)
    return np.cumsum(row_ptr).astype(np.int32), dst.astype(np.int32)


def csr_from_rows(rows, n):
    return csr_from_pairs(rows[:, 0], rows[:, 1], n)


def relerr(a, b):
    scale = np.abs(b).max(axis=0)
    return float((np.abs(a - b).max(axis=0) / np.where(scale > 0, scale, 1)).max())


def call(params, cells, row_ptr, col, n_entries=None, jkr=JKR):
    """One call through the C ABI on torch-owned device buffers; (status, dE/dq)."""
    import torch
    dev = torch.device("cuda", 0)
    n = cells.shape[0]
    ncols = cells.shape[1]
    d_cells = (torch.from_numpy(np.ascontiguousarray(cells.T)).to(dev) if n
               else torch.zeros(1, dtype=torch.float64, device=dev))
    d_rp = torch.from_numpy(np.ascontiguousarray(row_ptr, dtype=np.int32)).to(dev)
    d_col = torch.from_numpy(np.ascontiguousarray(col if len(col) else np.zeros(1), dtype=np.int32)).to(dev)
    d_out = torch.full((6, max(n, 1)), -7.0, dtype=torch.float64, device=dev)
    delta = np.ascontiguousarray(jkr[0])
    radius = np.ascontiguousarray(jkr[1])
    stream = torch.cuda.current_stream(dev)
    dp = ctypes.POINTER(ctypes.c_double)
    rc = abm_b200.LIB.abm_cell_cell_forces_noalloc(
        ctypes.byref(params), ctypes.c_void_p(d_cells.data_ptr()), n, ncols, max(n, 1),
        ctypes.c_void_p(d_rp.data_ptr()), ctypes.c_void_p(d_col.data_ptr()),
        len(col) if n_entries is None else n_entries,
        delta.ctypes.data_as(dp), radius.ctypes.data_as(dp), len(delta),
        ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, abm_b200.LIB.abm_noalloc_last_error().decode()
    status = abm_b200.LIB.abm_cell_cell_forces_noalloc_status(ctypes.c_void_p(stream.cuda_stream))
    return status, d_out.cpu().numpy().T[:n]


def oracle_forces(sim_params, cells, rows):
    o = orc.Oracle(sim_params, jkr=JKR)
    o.set_cells(cells)
    o.set_neighbors(rows)
    return o.cell_cell_forces()


def test_noalloc_forces_match_existing_entry_point_twice():
    # two calls in a row, on different states and sizes: the shared scratch array is reused
    for n, seed in ((6000, 41), (2500, 42)):
        cells = state(n, seed)
        sim = abm_b200.Simulation(cap_cells=n, jkr_table=JKR)
        sim.upload_cells(cells)
        sim.get_cell_neighbors()
        expect = sim.cell_cell_forces()
        row_ptr, col = csr_from_rows(sim.neighbors(), n)
        status, got = call(sim.params, cells, row_ptr, col)
        assert status == 0
        assert relerr(got, expect) <= RTOL_FP64
        sim.close()


@pytest.mark.parametrize("precision", [abm_b200.PRECISION_FP64, abm_b200.PRECISION_MIXED])
def test_noalloc_forces_match_oracle(precision):
    n = 5000
    cells = state(n, 43)
    sim = abm_b200.Simulation(cap_cells=n, jkr_table=JKR)
    sim.upload_cells(cells)
    sim.get_cell_neighbors()
    rows = sim.neighbors()
    sim.close()
    p, pd = abm_b200.make_params(cap_cells=n, precision=precision)
    expect = oracle_forces(pd, cells, rows)
    status, got = call(p, cells, *csr_from_rows(rows, n))
    assert status == 0
    err = relerr(got, expect)
    assert err <= (RTOL_FP64 if precision == abm_b200.PRECISION_FP64 else RTOL_MIXED), err


def test_noalloc_at_its_exact_limits():
    # 32768 cells and 524288 CSR entries: the true neighbor pairs plus pairs of cells far
    # apart (their force is exactly zero), so the result equals the oracle's
    n = MAX_CELLS
    cells = state(n, 44)
    sim = abm_b200.Simulation(cap_cells=n, jkr_table=JKR)
    sim.upload_cells(cells)
    sim.get_cell_neighbors()
    rows = sim.neighbors()
    sim.close()
    i, j = rows[:, 0].astype(np.int64), rows[:, 1].astype(np.int64)
    have = set((i * n + j).tolist())
    need = (MAX_ENTRIES - 2 * len(rows)) // 2
    assert need > 0
    rng = np.random.default_rng(9)
    r = cells[:, 1:4]
    reach = cells[:, 14].max() * 2 + 2 * 0.8
    extra = []
    while len(extra) < need:
        a, b = rng.integers(0, n, size=2)
        hi, lo = max(a, b), min(a, b)
        if hi == lo or (hi * n + lo) in have or np.linalg.norm(r[hi] - r[lo]) <= reach:
            continue
        have.add(hi * n + lo)
        extra.append((hi, lo))
    extra = np.array(extra)
    row_ptr, col = csr_from_pairs(np.concatenate([i, extra[:, 0]]), np.concatenate([j, extra[:, 1]]), n)
    assert len(col) == MAX_ENTRIES and row_ptr[-1] == MAX_ENTRIES
    p, pd = abm_b200.make_params(cap_cells=n)
    expect = oracle_forces(pd, cells, rows)
    status, got = call(p, cells, row_ptr, col)
    assert status == 0
    assert relerr(got, expect) <= RTOL_FP64


def test_noalloc_empty_call():
    p, _ = abm_b200.make_params(cap_cells=16)
    cells = np.zeros((0, 22))
    status, got = call(p, cells, np.zeros(1, dtype=np.int32), np.zeros(0, dtype=np.int32))
    assert status == 0 and got.shape == (0, 6)


def test_noalloc_rejects_a_bad_csr_on_the_device():
    n = 3000
    cells = state(n, 45)
    sim = abm_b200.Simulation(cap_cells=n, jkr_table=JKR)
    sim.upload_cells(cells)
    sim.get_cell_neighbors()
    rows = sim.neighbors()
    expect = sim.cell_cell_forces()
    sim.close()
    p, _ = abm_b200.make_params(cap_cells=n)
    row_ptr, col = csr_from_rows(rows, n)
    deg = np.diff(row_ptr)
    k = int(row_ptr[np.argmax(deg >= 1)])    # first entry of a row with neighbors
    bad_col = col.copy()
    bad_col[k] = n + 5                       # a column past the last cell
    short_ptr = row_ptr.copy()
    short_ptr[-1] -= 1                       # row_ptr[n] != n_entries
    unsorted = col.copy()
    a = int(row_ptr[np.argmax(deg >= 2)])    # a row with two neighbors or more
    unsorted[a], unsorted[a + 1] = unsorted[a + 1], unsorted[a]
    # a row whose first neighbor j0 is replaced by j0 - 1: the row stays sorted and in
    # range, but neither (r, j0 - 1) nor (j0, r) has its partner entry any more
    asym = col.copy()
    r = next(r for r in range(n) if row_ptr[r + 1] > row_ptr[r] and col[row_ptr[r]] >= 1
             and col[row_ptr[r]] - 1 != r)
    asym[row_ptr[r]] -= 1
    cases = [("column", row_ptr, bad_col), ("bounds", short_ptr, col), ("order", row_ptr, unsorted),
             ("symmetry", row_ptr, asym)]
    for what, rp, cl in cases:
        status, got = call(p, cells, rp, cl, n_entries=len(col))
        assert status == -1, what
        assert what in abm_b200.LIB.abm_noalloc_last_error().decode(), what
        assert np.isnan(got).all(), what
        # the next good call is unaffected
        status, got = call(p, cells, row_ptr, col)
        assert status == 0 and relerr(got, expect) <= RTOL_FP64


def test_noalloc_rejects_bad_arguments_on_the_host():
    lib = abm_b200.LIB
    dp = ctypes.POINTER(ctypes.c_double)
    delta = np.ascontiguousarray(JKR[0])
    radius = np.ascontiguousarray(JKR[1])
    flat = delta.copy()
    flat[10] = flat[9]

    def rc(params, n=8, n_entries=0, col=ctypes.c_void_p(1), d=delta):
        return lib.abm_cell_cell_forces_noalloc(ctypes.byref(params), ctypes.c_void_p(1), n, 22, n,
                                                ctypes.c_void_p(1), col, n_entries, d.ctypes.data_as(dp),
                                                radius.ctypes.data_as(dp), len(d), ctypes.c_void_p(1), None)
    p2, _ = abm_b200.make_params(cap_cells=16, **abm_b200.DEFAULTS_2D)
    assert rc(p2) == -1 and "3-D" in lib.abm_noalloc_last_error().decode()
    pa, _ = abm_b200.make_params(cap_cells=16, adhesion_mode=2)
    assert rc(pa) == -1 and "adhesion_mode" in lib.abm_noalloc_last_error().decode()
    p, _ = abm_b200.make_params(cap_cells=16)
    assert rc(p, d=flat) == -1 and "increasing" in lib.abm_noalloc_last_error().decode()
    assert rc(p, n_entries=4, col=None) == -1
    assert rc(p, n=0, n_entries=4) == -1
    assert rc(p, n=MAX_CELLS + 1) == -3 and "ABM_NOALLOC_MAX_CELLS" in lib.abm_noalloc_last_error().decode()
    assert rc(p, n_entries=MAX_ENTRIES + 1) == -3 and "ABM_NOALLOC_MAX_ENTRIES" in lib.abm_noalloc_last_error().decode()
