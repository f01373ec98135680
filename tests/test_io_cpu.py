"""Frame and lineage files of the C ABI against the reference's formats (restated in
oracle/io_ref.py from utils.hpp:96-311): byte for byte for the writers, round trips
for the readers, and the errors for bad input.  Host code, no GPU."""
import numpy as np
import pytest

import io_ref
from abm_b200 import frames, workloads


def state_3d(n=300, seed=4):
    cells, _ = workloads.biofilm_3d(n=n, seed=seed, disk_radius=40.0, p_contact=0.5)
    rng = np.random.default_rng(seed)
    cells[:, 0] = rng.permutation(n) + 7              # IDs
    cells[:, 15] = rng.uniform(0, 3, n)                # birth times
    cells[:, 16] = rng.normal(1.5, 0.1, n)
    cells[:, 20] = rng.integers(1, 3, n)               # groups
    cells[:5, 1] = [0.0, -0.0, 1e-7, -123456.789012345, 3.0e5]
    return cells


PARAMS = {"R": "0.8", "E0": "3900", "t_curr": "0.123456789", "dt_write": "0.01", "n_cells": "300"}


@pytest.mark.parametrize("extra", [None, {21: 1}, {21: 0}])
def test_write_cells_matches_the_reference_format(tmp_path, extra):
    cells = state_3d()
    path = tmp_path / "cells.txt"
    frames.write_cells(str(path), cells, PARAMS, extra_cols=extra)
    assert path.read_text() == io_ref.write_cells_text(cells, PARAMS, extra, dims=3)


def test_write_cells_2d_layout(tmp_path):
    cells = workloads.biofilm_2d(200, seed=2)
    cells[:, 16] = 2
    path = tmp_path / "cells2d.txt"
    frames.write_cells(str(path), cells, {"L0": "2"}, dims=2)
    assert path.read_text() == io_ref.write_cells_text(cells, {"L0": "2"}, None, dims=2)


def test_read_cells_round_trip(tmp_path):
    cells = state_3d()
    path = tmp_path / "cells.txt"
    frames.write_cells(str(path), cells, PARAMS, extra_cols={21: 1})
    back, params = frames.read_cells(str(path))
    assert params == PARAMS
    assert back.shape == (len(cells), 22)
    expect = np.array([[float("%.10g" % v) for v in row] for row in cells])
    expect[:, 0] = cells[:, 0].astype(int)
    expect[:, 20] = cells[:, 20].astype(int)
    assert np.array_equal(back, expect)
    # what was written at 10 digits reads back and writes out to the same bytes
    path2 = tmp_path / "again.txt"
    frames.write_cells(str(path2), back, params, extra_cols={21: 1})
    assert path2.read_bytes() == path.read_bytes()


def test_lineage_round_trip(tmp_path):
    parents = np.array([-1, -1, 0, 0, 1, 1, 2, 5, 5], dtype=np.int32)
    path = tmp_path / "lineage.txt"
    frames.write_lineage(str(path), parents)
    assert path.read_text() == io_ref.lineage_text(parents)
    assert np.array_equal(frames.read_lineage(str(path)), parents)


def test_empty_population_and_errors(tmp_path):
    path = tmp_path / "empty.txt"
    frames.write_cells(str(path), np.zeros((0, 22)), {"n_cells": "0"})
    assert path.read_text() == "# n_cells = 0\n"
    back, params = frames.read_cells(str(path))
    assert back.shape[0] == 0 and params == {"n_cells": "0"}
    with pytest.raises(RuntimeError, match="extra column"):
        frames.write_cells(str(path), state_3d(10), None, extra_cols={40: 1})
    with pytest.raises(RuntimeError, match="too few columns"):
        frames.write_cells(str(path), np.zeros((3, 10)), None)
    with pytest.raises(RuntimeError, match="cannot open"):
        frames.read_cells(str(tmp_path / "missing.txt"))


def test_read_cells_accepts_trailing_tabs_and_crlf(tmp_path):
    """readCells (utils.hpp:96-139) splits rows with std::getline(ss, token, '\\t'), which yields
    no empty token after a trailing tab, and std::stod ignores a trailing carriage return."""
    cells = state_3d(20)
    plain = tmp_path / "plain.txt"
    frames.write_cells(str(plain), cells, PARAMS)
    text = plain.read_text()
    odd = tmp_path / "odd.txt"
    odd.write_bytes("".join(line + ("\t\r\n" if not line.startswith("#") else "\r\n")
                            for line in text.splitlines()).encode())
    a, pa = frames.read_cells(str(plain))
    b, pb = frames.read_cells(str(odd))
    assert pa == pb and np.array_equal(a, b)
    bad = tmp_path / "bad.txt"
    bad.write_text("1\t\t2\n")
    with pytest.raises(RuntimeError, match="not a number"):
        frames.read_cells(str(bad))


def test_sparse_lineage_marks_absent_ids(tmp_path):
    path = tmp_path / "sparse.txt"
    path.write_text("0\t-1\n3\t0\n")
    assert list(frames.read_lineage(str(path))) == [-1, frames.ABSENT, frames.ABSENT, 0]


class FramesStandIn:
    """The calls write_frames and RunLog make on a Simulation, over host arrays: two
    frames of a growing population, the lineage, and the loop's counters."""

    def __init__(self):
        self.states = [state_3d(200, 5), state_3d(260, 6)]
        self.times, self.iters = [0.1, 0.2], [1000, 2150]
        self.lineage = np.arange(-1, 259, dtype=np.int32)
        self.counters = dict(iterations=2150, attempts=4400, retries=12, rebuilds=31, divisions=60, t=0.2,
                             dt=9.5e-5, last_max_error=0.42, n_cells=260, n_pairs=1900, rejected=11,
                             log_rows=0, cell_steps=512345)

    def frames_taken(self):
        return 2

    def download_frame(self, k):
        return self.states[k], self.times[k], self.iters[k], len(self.states[k])

    def parents(self):
        return self.lineage

    def stats(self):
        return dict(self.counters)


def test_run_log_lines_beside_the_frames(tmp_path):
    import json
    sim = FramesStandIn()
    ticks = iter([10.0, 12.5, 20.0])
    prefix = str(tmp_path / "run")
    with frames.RunLog(str(tmp_path / "run.jsonl"), clock=lambda: next(ticks)) as log:
        assert frames.write_frames(sim, prefix, PARAMS, log=log) == 2
        assert frames.write_frames(sim, prefix, PARAMS, start=2, log=log) == 2     # nothing new: no line
        sim.counters.update(iterations=2300, t=0.21)
        log.record(sim, note="end")
    lines = [json.loads(x) for x in open(str(tmp_path / "run.jsonl"))]
    assert len(lines) == 2
    first, last = lines
    # the reference's per-write fields (simulation.hpp:2035-2039) and the device counters
    assert first["iteration"] == 2150 and first["cells"] == 260 and first["t"] == 0.2 and first["dt"] == 9.5e-5
    assert first["time_elapsed_s"] == 2.5 and first["max_scaled_error"] == 0.42
    assert first["frames_written"] == 2 and first["rejected"] == 11 and first["cell_steps"] == 512345
    assert last["iteration"] == 2300 and last["time_elapsed_s"] == 7.5 and last["note"] == "end"
    # the frame files themselves are the reference's, with t_curr of each frame
    for k in range(2):
        cells, params = frames.read_cells("%s_iter%d.txt" % (prefix, sim.iters[k]))
        # ID through group (columns 0-20); gamma goes out only as a requested extra column
        assert cells.shape == (len(sim.states[k]), 21)
        assert np.array_equal(cells[:, [0, 20]], sim.states[k][:, [0, 20]])
        assert params["t_curr"] == "%.10g" % sim.times[k]
    assert np.array_equal(frames.read_lineage(prefix + "_lineage.txt"), sim.lineage[:260])
