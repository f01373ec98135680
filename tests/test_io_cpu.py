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
