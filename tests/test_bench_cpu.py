"""Host-side logic of bench.py that needs no GPU: argument aliases, the roofline
record (dominant group, algorithmic bytes, the ncu traffic looked up by group name),
the launch count and the byte model."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_cells_alias_and_defaults():
    a = bench.parse_args(["--cells", "1500"])
    assert a.n == 1500 and a.gpus == 1 and a.warmup >= 3
    assert bench.parse_args([]).n == 100_000


def test_roofline_takes_the_slowest_group_and_its_traffic():
    kernels = {"k_pair_pass(+proposal)": (18_000_000, 0.024), "k_attempt(proposal)": (34_400_000, 0.063)}
    r = bench.roofline(kernels, 0.43)
    assert r["kernel"] == "k_attempt(proposal)"
    assert abs(r["achieved"] - 34_400_000 / 0.063e-3 / 1e9) < 1e-6
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
        traffic = json.load(f)
    assert r["traffic"] == traffic["k_attempt(proposal)"]["bytes_per_launch"]
    assert set(r["other_kernels"]) == {"k_pair_pass(+proposal)"}


def test_every_group_name_has_a_traffic_entry():
    with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
        traffic = json.load(f)
    for name in ("k_pair_pass(+proposal)", "k_pair_pass", "k_attempt(proposal)", "k_attempt(trial+final)"):
        assert traffic[name]["bytes_per_launch"] > 0


def test_launch_count_follows_the_graph():
    t = {"iterations": 100, "retries": 3, "rejected": 2, "rebuilds": 1}
    # reference controller: pair pass, trial, final each iteration, plus the retries
    assert bench.launches("plain", t) == 300 + 3 + 18
    # learned: pair pass and trial; a failed proposal adds max_tries retries and the final
    assert bench.launches("chosen", t) == 200 + 2 * 4 + 18


def test_byte_model_per_cell():
    n, n_dir = 100_000, 1_506_000
    assert bench.attempt_bytes(n, False) == 224 * n
    assert bench.attempt_bytes(n, True) == 344 * n
    assert bench.pair_force_bytes(n, n_dir) == 120 * n + 4 * n_dir


def test_step_byte_model_worked_values():
    # B_step(s, P, E, K) at P = 10, E = 1, K = 100: ~962 B (Heun-Euler) and ~1762 B (BS3(2))
    assert abs(bench.step_byte_model(10, 1, 2) - 961.56) < 1e-9
    assert abs(bench.step_byte_model(10, 1, 4) - 1761.56) < 1e-9
    # each extra evaluation adds B_eval(s): 752 B and 1552 B
    assert abs(bench.step_byte_model(10, 2, 2) - bench.step_byte_model(10, 1, 2) - 752) < 1e-9


def test_rk_units_scale_by_the_error_test():
    import numpy as np
    cells = np.zeros((2, 22))
    cells[:, 1:7] = [[100.0, 0, 0, 1, 0, 0], [0, 0, 9.0, 0, 0, 1]]
    a = cells.copy()
    b = cells.copy()
    b[0, 1] += 1e-6          # tol (1 + 100) = 1.01e-6: 0.99 units
    b[1, 6] += 1e-9          # tol (1 + 1) = 2e-8: 0.05 units
    assert abs(bench.rk_units(a, b, cells) - 1e-6 / 1.01e-6) < 1e-8


def test_reference_arm_loads_no_product_library():
    # the reference arm builds its parameters from the package's structs and draws the
    # benchmark state with the oracle's build of the generator; the product library
    # never enters its process
    import subprocess
    code = (
        "import sys; sys.path[:0] = [%r, %r]\n"
        "import bench\n"
        "import abm_b200\n"
        "_, pd = abm_b200.make_params(cap_cells=8)\n"
        "cells, info = bench.workload(2000, 1, lib=bench.oracle_module().LIB)\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libabm_b200.so' not in maps, 'product library loaded'\n"
        "assert 'liboracle_abm.so' in maps\n"
        "print('ok', cells.shape)\n") % (ROOT, os.path.join(ROOT, "biofilm-abms_b200"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ok (2000, 22)" in r.stdout, r.stderr


def test_both_builds_of_the_generator_draw_the_same_state():
    # the benchmark state drawn by the package's library and by the oracle's build
    from abm_b200 import workloads
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import numpy as np
    import oracle_ref as orc
    a, ia = bench.workload(100_000, 1)
    b, ib = bench.workload(100_000, 1, lib=orc.LIB)
    assert np.array_equal(a, b) and ia == ib
    c = workloads.biofilm_2d(3000, seed=4)
    assert c.shape == (3000, 17)


def test_optimized_cpu_leg_runs_on_the_benchmark_state():
    # the context figure beside the faithful CPU run: same state and parameters, the
    # cell-list build and parallel pair forces; a small case of the same workload
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ref as orc
    args = bench.parse_args(["--cells", "3000"])
    cells, _ = bench.workload(args.n, 1, lib=orc.LIB)
    r = bench.cpu_optimized_rate(cells, args, 2, 2)
    assert r["value"] > 0 and r["cores"] == 2 and r["unit"] == bench.UNIT
    assert "2 accepted steps at n=3000" in r["sample"]
    json.dumps(r)
