"""abm_cell_cell_forces_noalloc: the cell-cell force entry point for callers that
cannot allocate device memory (their memory belongs to another allocator, or
they cannot take cudaMalloc's synchronisation in a step loop).  It must give the
same dE/dq as abm_cell_cell_forces on buffers the caller already owns, call after
call, with its scratch in the library's fixed device array.

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


def state(n, seed):
    cells, _ = workloads.biofilm_3d(n=n, seed=seed, disk_radius=300.0 * (n / 1e5) ** 0.5, p_contact=0.9)
    return cells


def csr_from_rows(rows, n):
    """Both directions of each (i, j) row, every row sorted ascending."""
    i = rows[:, 0].astype(np.int64)
    j = rows[:, 1].astype(np.int64)
    src = np.concatenate([i, j])
    dst = np.concatenate([j, i])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    row_ptr = np.zeros(n + 1, dtype=np.int32)
    np.add.at(row_ptr, src + 1, 1)
    return np.cumsum(row_ptr).astype(np.int32), dst.astype(np.int32)


def relerr(a, b):
    scale = np.abs(b).max(axis=0)
    return float((np.abs(a - b).max(axis=0) / np.where(scale > 0, scale, 1)).max())


def noalloc_forces(params, cells, row_ptr, col):
    import torch
    dev = torch.device("cuda", 0)
    n, ncols = cells.shape
    d_cells = torch.from_numpy(np.ascontiguousarray(cells.T)).to(dev)      # column-major n x ncols
    d_rp = torch.from_numpy(row_ptr).to(dev)
    d_col = torch.from_numpy(col if len(col) else np.zeros(1, np.int32)).to(dev)
    d_out = torch.zeros((6, n), dtype=torch.float64, device=dev)
    delta = np.ascontiguousarray(JKR[0])
    radius = np.ascontiguousarray(JKR[1])
    stream = torch.cuda.current_stream(dev)
    dp = ctypes.POINTER(ctypes.c_double)
    rc = abm_b200.LIB.abm_cell_cell_forces_noalloc(
        ctypes.byref(params), ctypes.c_void_p(d_cells.data_ptr()), n, ncols, n,
        ctypes.c_void_p(d_rp.data_ptr()), ctypes.c_void_p(d_col.data_ptr()), len(col),
        delta.ctypes.data_as(dp), radius.ctypes.data_as(dp), len(delta),
        ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, abm_b200.LIB.abm_noalloc_last_error().decode()
    stream.synchronize()
    return d_out.cpu().numpy().T


def test_noalloc_forces_match_existing_entry_point_twice():
    # two calls in a row, on different states and sizes: the shared scratch array is reused
    for n, seed in ((6000, 41), (2500, 42)):
        cells = state(n, seed)
        sim = abm_b200.Simulation(cap_cells=n, jkr_table=JKR)
        sim.upload_cells(cells)
        sim.get_cell_neighbors()
        expect = sim.cell_cell_forces()
        row_ptr, col = csr_from_rows(sim.neighbors(), n)
        got = noalloc_forces(sim.params, cells, row_ptr, col)
        assert relerr(got, expect) <= 1e-10
        sim.close()


def test_noalloc_rejects_sizes_beyond_the_limit():
    p, _ = abm_b200.make_params(cap_cells=16)
    n = 32769
    rc = abm_b200.LIB.abm_cell_cell_forces_noalloc(
        ctypes.byref(p), ctypes.c_void_p(1), n, 22, n, ctypes.c_void_p(1), ctypes.c_void_p(1), 0,
        None, None, 0, ctypes.c_void_p(1), None)
    assert rc == -3
    assert "ABM_NOALLOC_MAX_CELLS" in abm_b200.LIB.abm_noalloc_last_error().decode()
