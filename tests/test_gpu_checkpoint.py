"""Exact binary checkpoints (abm_save_checkpoint / abm_load_checkpoint).

The reference resumes a run from its text frames (readCells and readLineage,
utils.hpp:96-139 and 265-287 of both models), whose 10 significant digits move the
resumed run off the course of the uninterrupted one.  A checkpoint keeps the FP64
cells, the neighbor set, the lineage, the clock and the controllers' history, so a
run saved at iteration k and resumed in a new context ends bit for bit where the
uninterrupted run ends: divisions, periodic rebuilds and, under the learned and PI
controllers, the proposals that read the history, included.
"""
import os

import numpy as np
import pytest

import abm_b200
from abm_b200 import stepsize, workloads
import oracle_ref as orc

pytestmark = pytest.mark.gpu

JKR = orc.jkr_table(0.8, 0.5, 3900.0, 100.0, 100)
DIV_KW = dict(growth_mean=1.5, growth_std=0.1, daughter_length_std=0.05, daughter_angle_xy_bound=0.3,
              daughter_angle_z_bound=0.1, rng_seed=7)
STATS = ("iterations", "attempts", "retries", "rejected", "divisions", "rebuilds")


def growing_state(n, seed):
    """A patch of the benchmark's density whose cells grow, 30 of them about to divide."""
    cells, _ = workloads.biofilm_3d(n=n, seed=seed, disk_radius=300.0 * np.sqrt(n / 100000.0), p_contact=0.9)
    rng = np.random.default_rng(seed)
    cells[:, 13] = rng.uniform(4.5, 5.55, size=n)
    cells[:30, 13] = 5.6 - rng.uniform(0.0, 2e-3, size=30)
    cells[:, 14] = cells[:, 13] / 2
    cells[:, 16] = rng.normal(1.5, 0.1, size=n)
    return cells


def new_sim(cells, controller, cap=None):
    sim = abm_b200.Simulation(jkr_table=JKR, cap_cells=cap or 3 * len(cells), max_stepsize=1e-3,
                              iter_update_neighbors=10, controller=controller, **DIV_KW)
    if controller == abm_b200.CONTROLLER_LEARNED:
        sim.set_stepsize_weights(stepsize.load())
    return sim


def start(cells, controller):
    sim = new_sim(cells, controller)
    sim.upload_cells(cells)
    sim.set_parents(-np.ones(len(cells), dtype=np.int32))
    sim.set_clock(0.0, 1e-4, 0)
    sim.get_cell_neighbors()
    return sim


def end_state(sim, s):
    return sim.download_cells(), sim.parents(), sim.clock(), s


@pytest.mark.parametrize("controller", [abm_b200.CONTROLLER_REFERENCE, abm_b200.CONTROLLER_LEARNED,
                                        abm_b200.CONTROLLER_PI])
def test_resumed_run_ends_bit_for_bit_where_the_uninterrupted_run_ends(controller, tmp_path):
    cells = growing_state(400, 35)
    # uninterrupted: 35 iterations (rebuilds every 10, divisions along the way)
    a = start(cells, controller)
    ref = end_state(a, a.iterate(35))
    a.close()
    # 17 iterations, checkpoint, then 18 more in a context that starts from the file
    b = start(cells, controller)
    b.iterate(17)
    path = os.fspath(tmp_path / "run.ckpt")
    b.save_checkpoint(path)
    mid_cells, mid_clock = b.download_cells(), b.clock()
    b.close()
    c = new_sim(cells, controller)
    c.load_checkpoint(path)
    assert np.array_equal(c.download_cells(), mid_cells) and c.clock() == mid_clock
    got = end_state(c, c.iterate(18))
    c.close()
    (ca, pa, ta, sa), (cb, pb, tb, sb) = ref, got
    assert sa["divisions"] > 0 and sa["rebuilds"] > 3
    assert ta == tb
    assert np.array_equal(pa, pb)
    assert ca.shape == cb.shape and np.array_equal(ca, cb)
    for k in STATS:
        assert sa[k] == sb[k], k


def test_checkpoint_rejects_what_it_cannot_resume(tmp_path):
    cells = growing_state(300, 36)
    sim = start(cells, abm_b200.CONTROLLER_REFERENCE)
    sim.iterate(3)
    path = os.fspath(tmp_path / "run.ckpt")
    sim.save_checkpoint(path)
    blob = open(path, "rb").read()
    # header: magic, then dims, ncols, n, pairs, lineage length, 0
    head = np.frombuffer(blob[8:32], dtype=np.int32)
    n = sim.num_cells()
    assert blob[:8] == b"ABMCKP01" and head[0] == 3 and head[2] == n and head[4] == len(sim.parents())
    before = sim.download_cells()

    def rejected(data, sim_kw=None, cap=None):
        p = os.fspath(tmp_path / "bad.ckpt")
        with open(p, "wb") as f:
            f.write(data)
        s = abm_b200.Simulation(**sim_kw) if sim_kw else new_sim(cells, abm_b200.CONTROLLER_REFERENCE, cap=cap)
        with pytest.raises(RuntimeError) as e:
            s.load_checkpoint(p)
        s.close()
        return str(e.value)

    assert "ABM_ERR_ARG" in rejected(blob[:-4])                    # truncated
    assert "ABM_ERR_ARG" in rejected(blob + b"\0")                 # trailing bytes
    assert "ABM_ERR_ARG" in rejected(b"ABMCKP00" + blob[8:])        # another format
    assert "ABM_ERR_CAPACITY" in rejected(blob, cap=n - 1)
    msg = rejected(blob, sim_kw=dict(cap_cells=2 * n, **abm_b200.DEFAULTS_2D))
    assert "ABM_ERR_ARG" in msg and "other model" in msg
    # saving before the neighbor set exists is a call-order error
    fresh = new_sim(cells, abm_b200.CONTROLLER_REFERENCE)
    fresh.upload_cells(cells)
    with pytest.raises(RuntimeError) as e:
        fresh.save_checkpoint(os.fspath(tmp_path / "early.ckpt"))
    assert "ABM_ERR_STATE" in str(e.value)
    fresh.close()
    # a rejected load leaves nothing behind: a good one then resumes the saved state
    bad = os.fspath(tmp_path / "truncated.ckpt")
    with open(bad, "wb") as f:
        f.write(blob[: len(blob) // 2])
    c = new_sim(cells, abm_b200.CONTROLLER_REFERENCE)
    with pytest.raises(RuntimeError):
        c.load_checkpoint(bad)
    c.load_checkpoint(path)
    assert np.array_equal(c.download_cells(), before)
    assert c.clock() == sim.clock()
    c.close()
    sim.close()
