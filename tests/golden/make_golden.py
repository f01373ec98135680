"""Generate golden vectors from the reference's own known-answer tests.

The reference's Catch2 tests cannot be compiled here (no Eigen/CGAL/Catch2),
so this script reads their source text and evaluates the literal inputs and
expected outputs of every `testDistBetweenCells(...)` and
`testNearestCellBodyCoordToPoint(...)` call:

  ABM-3d/ABM-3d-cpp/test/src/testDistBetweenCells.cpp:143-506
  ABM-2d/ABM-2d-cpp/test/src/testDistBetweenCells.cpp:85-344

Statements inside each TEST_CASE body are translated line by line into Python
(double arithmetic is IEEE binary64 in both languages).  The reference's own
line-to-line helper `distBetweenLines` (Vega & Lago 1994, testDistBetweenCells.cpp
3D:42-53) is restated below because one 3-D case uses it to form its target.

Run in a container that has the reference checked out:
    python tests/golden/make_golden.py /path/to/reference
It writes dist3d_cases.json and dist2d_cases.json next to itself.  The
tolerance asserted by the reference for all of these cases is 1e-8 (absolute).
"""
import json
import math
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def dist_between_lines(r1, n1, r2, n2):
    """Shortest vector between two infinite lines (testDistBetweenCells.cpp:42-53)."""
    dot = lambda a, b: (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]
    r12 = [r2[k] - r1[k] for k in range(3)]
    c = dot(n1, n2)
    s = (dot(r12, n1) - c * dot(r12, n2)) / (1.0 - c * c)
    t = (-dot(r12, n2) + c * dot(r12, n1)) / (1.0 - c * c)
    d = [r12[k] + t * n2[k] - s * n1[k] for k in range(3)]
    return (d, s, t)


def _strip_comments(src):
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def _test_case_bodies(src):
    bodies = []
    for m in re.finditer(r"TEST_CASE\(\s*\"[^\"]*\"\s*,\s*\"[^\"]*\"\s*\)\s*\{", src):
        depth, k = 1, m.end()
        while depth:
            depth += {"{": 1, "}": -1}.get(src[k], 0)
            k += 1
        bodies.append(src[m.end():k - 1])
    return bodies


def _py_expr(expr):
    e = expr.strip()
    e = re.sub(r"boost::math::constants::sixth_pi<T>\(\)", "(math.pi/6)", e)
    e = re.sub(r"boost::math::constants::pi<T>\(\)", "math.pi", e)
    e = re.sub(r"std::get<(\d)>\((\w+)\)\((\d)\)", r"\2[\1][\3]", e)
    e = re.sub(r"std::get<(\d)>\((\w+)\)", r"\2[\1]", e)
    e = re.sub(r"\b(sin|cos|tan|sqrt)\(", r"math.\1(", e)
    if re.search(r"(?<![\w.])\d+\s*/\s*\d+(?![\w.])", e):
        raise ValueError("integer division in reference expression: " + expr)
    return e


def _split_args(s):
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
            continue
        depth += ch == "("
        depth -= ch == ")"
        cur += ch
    out.append(cur)
    return [a for a in (x.strip() for x in out) if a]


def extract(path, dim):
    src = _strip_comments(open(path).read())
    nearest, dists = [], []
    for body in _test_case_bodies(src):
        env = {"math": math, "distBetweenLines": dist_between_lines}
        for stmt in body.split(";"):
            st = " ".join(stmt.split())
            if not st:
                continue
            m = re.match(r"(testDistBetweenCells|testNearestCellBodyCoordToPoint)\s*\((.*)\)$", st)
            if m:
                vals = [float(eval(_py_expr(a), env)) for a in _split_args(m.group(2))]
                (dists if m.group(1) == "testDistBetweenCells" else nearest).append(vals)
                continue
            m = re.match(r"(?:Matrix<T, \d, 1>|T|auto)?\s*(\w+)\s*<<\s*(.*)$", st)
            if m and "<<" in st:
                env[m.group(1)] = [float(eval(_py_expr(a), env)) for a in _split_args(m.group(2))]
                continue
            m = re.match(r"(?:T|auto)\s+(\w+)\s*=\s*(.*)$", st) or re.match(r"(\w+)\s*=\s*(.*)$", st)
            if m:
                env[m.group(1)] = eval(_py_expr(m.group(2)), env)
                continue
            if re.match(r"(T|Matrix<T, \d, 1>|K)\s+[\w, ]+$", st):
                continue   # declarations without initialisers
            raise ValueError("untranslated statement in %s: %s" % (path, st))
    cases = []
    for v in dists:
        if dim == 3:
            r1, n1, h1, r2, n2, h2 = v[0:3], v[3:6], v[6], v[7:10], v[10:13], v[13]
            d, s, t = v[14:17], v[17], v[18]
        else:
            r1, n1, h1, r2, n2, h2 = v[0:2], v[2:4], v[4], v[5:7], v[7:9], v[9]
            d, s, t = v[10:12], v[12], v[13]
        cases.append({"r1": r1, "n1": n1, "half_l1": h1, "r2": r2, "n2": n2, "half_l2": h2,
                      "d": d, "s": s, "t": t})
    near = []
    for v in nearest:
        k = dim
        near.append({"r": v[0:k], "n": v[k:2 * k], "half_l": v[2 * k], "q": v[2 * k + 1:3 * k + 1],
                     "target": v[3 * k + 1]})
    return {"source": os.path.relpath(path, REF) if REF else path, "tolerance_abs": 1e-8,
            "dist_cases": cases, "nearest_cases": near}


REF = None

if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <path of a kmnam/biofilm-ABMs checkout>")
    REF = sys.argv[1]
    for dim, rel in ((3, "ABM-3d/ABM-3d-cpp/test/src/testDistBetweenCells.cpp"),
                     (2, "ABM-2d/ABM-2d-cpp/test/src/testDistBetweenCells.cpp")):
        out = extract(os.path.join(REF, rel), dim)
        with open(os.path.join(HERE, "dist%dd_cases.json" % dim), "w") as f:
            json.dump(out, f, indent=1)
        print("dim %d: %d distance cases, %d nearest-point cases" %
              (dim, len(out["dist_cases"]), len(out["nearest_cases"])))
