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
