"""Frames of the device-resident loop (runSimulation's dt_write writes,
simulation.hpp:2025-2058): the ring snapshots taken inside graph-launched iterations
are the states of exactly the steps whose time crosses a multiple of dt_write, bit
for bit, and write_frames writes them in the reference's file formats."""
import math

import numpy as np
import pytest

import abm_b200
import io_ref
from abm_b200 import frames, stepsize

pytestmark = pytest.mark.gpu


def colony():
    cells = stepsize.growing_colony(600, 3)
    rng = np.random.default_rng(3)
    cells[:30, 13] = 5.6 - rng.uniform(0.0, 2e-4, size=30)       # about to reach Ldiv: divisions early
    cells[:30, 14] = cells[:30, 13] / 2
    kw = dict(stepsize.GROWTH_KW, max_stepsize=1e-3, iter_update_neighbors=10, rng_seed=11)
    return cells, kw


def start(cells, kw):
    sim = abm_b200.Simulation(cap_cells=4 * len(cells), **kw)
    sim.upload_cells(cells)
    sim.set_parents(-np.ones(len(cells), dtype=np.int32))
    sim.set_clock(0.0, 1e-4, 0)
    sim.get_cell_neighbors()
    return sim


def stepped(cells, kw, iters):
    """The run one iteration at a time: (iteration, t, dt, cells, lineage length) after each."""
    b = start(cells, kw)
    rec = []
    for _ in range(iters):
        b.iterate(1)
        t, dt, it = b.clock()
        rec.append((it, t, dt, b.download_cells(), len(b.parents())))
    parents = np.asarray(b.parents())
    assert b.stats()["divisions"] > 0
    b.close()
    return rec, parents


def crossings(rec, dt_write):
    # simulation.hpp:2025-2028
    return [r for r in rec if math.fmod(r[1] - r[2] + 1e-12, dt_write) > math.fmod(r[1] + 1e-12, dt_write)]


def test_frames_are_the_states_of_the_crossing_steps(tmp_path):
    cells, kw = colony()
    iters = 60
    rec, parents = stepped(cells, kw, iters)
    # a few steps per frame: the step size varies by orders of magnitude along the run
    dt_write = 2.5 * float(np.median([r[2] for r in rec]))
    expect = crossings(rec, dt_write)
    assert len(expect) > 2
    a = start(cells, kw)
    a.set_frames(dt_write, slots=64)
    a.iterate(iters)                                # graph launches, several iterations each
    assert a.frames_taken() == len(expect)
    for k, (it, t, dt, c, npar) in enumerate(expect):
        fc, ft, fit, fnp = a.download_frame(k)
        assert (fit, ft, fnp) == (it, t, npar)
        assert np.array_equal(fc, c)
    # files as runSimulation writes them
    prefix = str(tmp_path / "run")
    params = {"R": "0.8", "dt_write": "%.10g" % dt_write}
    assert frames.write_frames(a, prefix, params) == len(expect)
    it, t, dt, c, npar = expect[-1]
    text = (tmp_path / ("run_iter%d.txt" % it)).read_text()
    assert text == io_ref.write_cells_text(c, dict(params, t_curr="%.10g" % t), None, dims=3)
    assert np.array_equal(frames.read_lineage(prefix + "_lineage.txt"), parents[:npar])
    a.close()


def test_ring_overwrite_is_reported_and_frames_turn_off():
    cells, kw = colony()
    rec, _ = stepped(cells, kw, 40)
    a = start(cells, kw)
    a.set_frames(1.5 * float(np.median([r[2] for r in rec])), slots=2)
    a.iterate(40)
    taken = a.frames_taken()
    assert taken > 2
    with pytest.raises(RuntimeError, match="overwritten"):
        a.download_frame(0)
    a.download_frame(taken - 1)
    a.set_frames(0.0, 0)
    a.iterate(10)
    assert a.frames_taken() == 0
    a.close()
