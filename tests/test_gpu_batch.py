"""Batches: independent contexts advanced by one graph launch per iteration.
A context in a batch must end bit for bit where it ends when advanced alone
(same kernels, same arithmetic, its own clock, step size, RNG counters and
division events); the device cell limit must stop a context at its target; the
autotuner must return a valid pair-kernel tile."""
import numpy as np
import pytest

import abm_b200
from abm_b200 import replicates, workloads
import oracle_ref as orc

pytestmark = pytest.mark.gpu
JKR = orc.jkr_table(0.8, 0.5, 3900.0, 100.0, 100)


def ctx_2d(cells, seed, **kw):
    p = dict(replicates.CONFIG0, cap_cells=3 * len(cells) + 64, rng_seed=seed, max_stepsize=1e-3,
             iter_update_neighbors=10)
    p.update(kw)
    s = abm_b200.Simulation(**p)
    s.upload_cells(cells)
    s.set_parents(-np.ones(len(cells), dtype=np.int32))
    s.set_clock(0.0, p["max_stepsize"], 0)
    return s


def ctx_3d(cells):
    s = abm_b200.Simulation(cap_cells=len(cells) + 16, jkr_table=JKR, iter_update_neighbors=10, max_stepsize=1e-5)
    s.upload_cells(cells)
    return s


def states():
    a = replicates.start_state(300, 1)
    b = replicates.start_state(700, 2)
    c = replicates.start_state(1500, 3)
    for x in (a, b, c):
        x[:25, 9] = 4.4 - 1e-4          # about to reach Ldiv: divisions within the run
        x[:25, 10] = x[:25, 9] / 2
    d, _ = workloads.biofilm_3d(n=1200, seed=4, disk_radius=300.0 * np.sqrt(1200 / 1e5), p_contact=0.9)
    return a, b, c, d


def test_batch_matches_contexts_advanced_alone():
    a, b, c, d = states()
    alone = [ctx_2d(a, 11), ctx_2d(b, 12), ctx_2d(c, 13, integration_mode=1), ctx_3d(d)]
    batched = [ctx_2d(a, 11), ctx_2d(b, 12), ctx_2d(c, 13, integration_mode=1), ctx_3d(d)]
    for s in alone + batched:
        s.get_cell_neighbors()
    for s in alone:
        s.iterate(45)
    bt = abm_b200.Batch(batched)
    bt.iterate(45)
    bt.synchronize()
    divided = 0
    for s1, s2 in zip(alone, batched):
        c1, c2 = s1.download_cells(), s2.download_cells()
        assert c1.shape == c2.shape
        assert np.array_equal(c1, c2)
        assert s1.clock() == s2.clock()
        st1, st2 = s1.stats(), s2.stats()
        for k in ("iterations", "attempts", "retries", "rebuilds", "divisions", "rejected", "cell_steps"):
            assert st1[k] == st2[k], k
        assert np.array_equal(s1.neighbors(), s2.neighbors())
        if s1.dims == 2:
            assert np.array_equal(s1.parents(), s2.parents())
        divided += st1["divisions"]
    assert divided > 0
    bt.close()


def test_batch_cell_limit_stops_each_replicate():
    targets = [8, 20, 33]
    bt, sims = replicates.make_batch(targets, seed=5, founders=True, max_stepsize=1e-3, iter_update_neighbors=50)
    for _ in range(40):
        bt.iterate(250)
        bt.synchronize()
        if all(s.num_cells() >= t for s, t in zip(sims, targets)):
            break
    for s, t in zip(sims, targets):
        n = s.num_cells()
        assert t <= n < 2 * t
        clock = s.clock()
        cells = s.download_cells()
        st = s.stats()
        assert np.all(np.isfinite(cells))
        assert st["cell_steps"] > 0
    # halted replicates do not move: no further iterations, cells unchanged
    bt.iterate(20)
    bt.synchronize()
    it0 = [s.stats()["iterations"] for s in sims]
    before = [s.download_cells() for s in sims]
    bt.iterate(20)
    bt.synchronize()
    for s, c0, i0 in zip(sims, before, it0):
        assert np.array_equal(s.download_cells(), c0)
        assert s.stats()["iterations"] == i0
    bt.close()


def test_autotuner_picks_a_pair_tile():
    cells = replicates.start_state(5000, 9)
    best, times = abm_b200.autotune_pair_tile(cells, launches=5, **{k: v for k, v in replicates.CONFIG0.items()})
    assert best[0] in (512, 1024, 2048) and best[1] in (1, 2, 4)
    assert len(times) == 9 and all(t > 0 for t in times.values())
    assert times[best] == min(times.values())


def test_pair_tile_shapes_give_the_same_forces():
    cells = replicates.start_state(3000, 10)
    out = []
    for tile, bpsm in ((512, 1), (1024, 2), (2048, 4)):
        s = abm_b200.Simulation(cap_cells=3100, pair_tile=tile, pair_blocks_per_sm=bpsm,
                                **{k: v for k, v in replicates.CONFIG0.items()})
        s.upload_cells(cells)
        s.get_cell_neighbors()
        out.append(s.cell_cell_forces())
        s.close()
    # each cell's sum runs over its CSR row in a fixed order: the tile shape changes nothing
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[1], out[2])
