"""Frame and lineage files in the reference's text formats (writeCells / readCells /
writeLineage / readLineage, utils.hpp:96-311), through the C ABI (abm_write_cells,
abm_read_cells, abm_write_lineage, abm_read_lineage)."""
import ctypes
import os

import numpy as np

from . import LIB

_c_int_p = ctypes.POINTER(ctypes.c_int)
LIB.abm_write_cells.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.c_char_p, _c_int_p, _c_int_p, ctypes.c_int]
LIB.abm_read_cells.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _c_int_p, _c_int_p,
                               ctypes.c_char_p, ctypes.c_int]
LIB.abm_write_lineage.argtypes = [ctypes.c_char_p, _c_int_p, ctypes.c_int]
LIB.abm_read_lineage.argtypes = [ctypes.c_char_p, _c_int_p, ctypes.c_int, _c_int_p]
LIB.abm_io_last_error.restype = ctypes.c_char_p
for _f in (LIB.abm_write_cells, LIB.abm_read_cells, LIB.abm_write_lineage, LIB.abm_read_lineage):
    _f.restype = ctypes.c_int


def _check(rc, what):
    if rc != 0:
        raise RuntimeError("%s failed (%d): %s" % (what, rc, LIB.abm_io_last_error().decode()))


def params_text(params):
    """"key = value" lines: a dict in sorted key order (the reference keeps its
    parameters in a std::map), or a sequence of (key, value) pairs in its order."""
    items = sorted(params.items()) if isinstance(params, dict) else list(params or [])
    return "".join("%s = %s\n" % (k, v) for k, v in items)


def write_cells(path, cells, params=None, extra_cols=None, dims=3):
    """writeCells: `extra_cols` maps column -> 0 (integer) or 1 (double), like the
    reference's write_other_cols."""
    a = np.asfortranarray(cells, dtype=np.float64)
    n, ncols = a.shape
    ec = sorted((extra_cols or {}).items())
    cols = (ctypes.c_int * max(len(ec), 1))(*[c for c, _ in ec])
    types = (ctypes.c_int * max(len(ec), 1))(*[t for _, t in ec])
    _check(LIB.abm_write_cells(os.fsencode(path), a.ctypes.data, n, ncols, max(n, 1), dims,
                               params_text(params).encode(), cols, types, len(ec)), "abm_write_cells")


def read_cells(path):
    """readCells: (cells (n, ncols) float64 Fortran order, params dict of strings)."""
    p = os.fsencode(path)
    n, nc = ctypes.c_int(), ctypes.c_int()
    _check(LIB.abm_read_cells(p, None, 0, 0, ctypes.byref(n), ctypes.byref(nc), None, 0), "abm_read_cells")
    cells = np.zeros((n.value, nc.value), dtype=np.float64, order="F")
    size = os.path.getsize(path) + 1
    buf = ctypes.create_string_buffer(size)
    _check(LIB.abm_read_cells(p, cells.ctypes.data if cells.size else None, max(n.value, 1), max(nc.value, 1),
                              ctypes.byref(n), ctypes.byref(nc), buf, size), "abm_read_cells")
    params = dict(line.split(" = ", 1) for line in buf.value.decode().splitlines() if " = " in line)
    return cells, params


def write_lineage(path, parents):
    """writeLineage: "i<TAB>parents[i]" lines."""
    a = np.ascontiguousarray(parents, dtype=np.int32)
    _check(LIB.abm_write_lineage(os.fsencode(path), a.ctypes.data_as(_c_int_p), len(a)), "abm_write_lineage")


ABSENT = -2   # an ID the lineage file does not list (-1 is the parent of an initial cell)


def read_lineage(path):
    """readLineage (utils.hpp:265-287): parents indexed by cell ID.  The reference returns a map;
    IDs below the largest one that the file does not list read as ABSENT."""
    p = os.fsencode(path)
    n = ctypes.c_int()
    _check(LIB.abm_read_lineage(p, None, 0, ctypes.byref(n)), "abm_read_lineage")
    out = np.full(n.value, ABSENT, dtype=np.int32)
    _check(LIB.abm_read_lineage(p, out.ctypes.data_as(_c_int_p), len(out), ctypes.byref(n)), "abm_read_lineage")
    return out


def write_frames(sim, outprefix, params=None, start=0, extra_cols=None, dims=3, log=None):
    """Write frames start .. taken-1 of a Simulation with frames on, as runSimulation
    writes at its dt_write crossings (simulation.hpp:2045-2058): "<outprefix>_iter<i>.txt"
    with the parameters plus t_curr, then "<outprefix>_lineage.txt" with the lineage up
    to the last frame written.  With a RunLog `log`, one line of the loop's state and
    counters follows the files.  Returns the index of the next frame to write."""
    taken = sim.frames_taken()
    params = dict(params or {})
    n_parents = None
    for k in range(start, taken):
        cells, t, it, n_parents = sim.download_frame(k)
        params["t_curr"] = "%.10g" % t                 # floatToString(t), simulation.hpp:66-72
        write_cells("%s_iter%d.txt" % (outprefix, it), cells, params, extra_cols, dims)
    if n_parents is not None:
        write_lineage("%s_lineage.txt" % outprefix, np.asarray(sim.parents())[:n_parents])
    if log is not None and taken > start:
        log.record(sim, frames_written=taken - start)
    return taken


class RunLog:
    """One JSON line per frame write, in place of the line runSimulation prints there
    (simulation.hpp:2030-2039: iteration, cells, time, time elapsed since the last write,
    dt).  The reference also prints the max and mean absolute RK error of the last step;
    the device keeps the scaled max error E of the accepted attempt instead, logged as
    `max_scaled_error`.  The loop's counters (attempts, retries, rejected first attempts,
    rebuilds, divisions, neighbor pairs, cell-steps) come with each line, so a run's
    controller behaviour can be read back without re-running it.

    `sim` is anything with a `stats()` method returning the abm_stats fields as a dict
    (abm_b200.Simulation does).  Lines are appended and flushed as they are written."""

    def __init__(self, path, clock=None):
        import time
        self._clock = clock or time.monotonic
        self._last = self._clock()
        self._f = open(path, "a")

    def record(self, sim, **extra):
        """Append the line for the state `sim` is in now; `extra` keys go into it as given."""
        import json
        s = sim.stats()
        now = self._clock()
        line = {"iteration": int(s["iterations"]), "cells": int(s["n_cells"]), "t": float(s["t"]),
                "time_elapsed_s": now - self._last, "dt": float(s["dt"]),
                "max_scaled_error": float(s["last_max_error"])}
        for k in ("attempts", "retries", "rejected", "rebuilds", "divisions", "n_pairs", "cell_steps"):
            line[k] = int(s[k])
        line.update(extra)
        self._last = now
        self._f.write(json.dumps(line) + "\n")
        self._f.flush()
        return line

    def close(self):
        if self._f:
            self._f.close()
            self._f = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
