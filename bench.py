#!/usr/bin/env python
"""Benchmark: accepted cell-steps/s of the 3-D mechanics step at 100k cells,
chosen configuration vs the plain FP64 GPU path at equal RK tolerance.

Workload (one "step" = one accepted iteration of the runSimulation loop body,
ABM-3d/ABM-3d-cpp/include/simulation.hpp:1617-1864): 100,000 cells, centres
uniform in a 300 um disk with z in [R, 10] um, no growth or division, Heun-Euler
2(1) (the 3-D driver's default), RK tolerance 1e-8, dt capped at 1e-6 h,
isotropic JKR cell-cell adhesion (gamma = 100) and cell-surface Hertz + JKR.
Inputs are seeded synthetic states (no dataset is involved).

  chosen    mixed precision (segment distance and pair force in FP32, the rest
            FP64) and the learned step-size controller (the network's proposal is
            one RK attempt, accepted when its embedded error passes)
  plain     FP64 everywhere with the reference controller (trial + final re-run)

  value     chosen: device-resident throughput, CUDA events on the context stream,
            L2 flushed (256 MB write) between timed steps, max over ranks;
            `plain` holds the same figures for the plain path
  e2e       through the C ABI with pinned host buffers: upload cells -> one
            iteration -> download cells, every step
  roofline  the dominant kernel's algorithmic bytes per launch / its
            event-timed duration, against MEASURED_PEAKS.json
  cpu_baseline / --impl reference
            the oracle (a C++ restatement of the reference path, run the way
            the reference runs it: O(n^2) neighbor build, serial pair loops,
            pair forces recomputed per stage, OpenMP on the per-cell loops)

Multi-GPU: replicas only (each rank advances its own biofilm; no collective on
the data path), scaling "weak".
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "biofilm-abms_b200"))

METRIC = "accepted cell-steps/s @100k 3D cells"
UNIT = "cell-steps/s"
N_CELLS = 100_000
SEED = 1
P_CONTACT = 0.9
FLUSH_BYTES = 256 << 20
BINDING_MAX_DT = 1e-4      # h: a cap that the error test, not the cap, binds at


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", "--cells", dest="n", type=int, default=N_CELLS)
    ap.add_argument("--tableau", type=int, default=1, help="1 HE21, 2 BS32, 3 RKF45, 4 DP54")
    ap.add_argument("--variant", default="chosen", choices=["chosen", "plain"],
                    help="headline configuration; the other one is timed beside it unless --only")
    ap.add_argument("--only", action="store_true", help="time the headline variant only")
    ap.add_argument("--workload", default="3d", choices=["3d", "replicates", "growth"],
                    help="3d: the 100k-cell headline; replicates: batched 2-D replicate biofilms; "
                         "growth: 3-D growth from one founder cell, plain vs chosen")
    ap.add_argument("--growth-target", type=int, default=200_000)
    ap.add_argument("--growth-max-dt", type=float, default=1e-4, help="max_stepsize of the growth run (h)")
    ap.add_argument("--growth-max-seconds", type=float, default=600.0,
                    help="stop an arm of the growth run after this much device time")
    ap.add_argument("--growth-arms", default="plain,chosen", help="arms of the growth run")
    ap.add_argument("--weights", default=None, help="step-size network weights (.npz); default: the shipped ones")
    ap.add_argument("--replicates", type=int, default=256)
    ap.add_argument("--replicate-start", default="founder", choices=["founder", "near-target"],
                    help="replicates grow from one founder cell each (the configuration), or start at 90 %% "
                         "of their targets")
    ap.add_argument("--lanes", type=int, default=8)
    ap.add_argument("--tile", type=int, default=0, help="screened pair pass: CSR entries per block tile")
    ap.add_argument("--bpsm", type=int, default=0, help="screened pair pass: blocks per SM")
    ap.add_argument("--pair-sum", type=int, default=0, help="1: shares summed in the first attempt, 2: separately")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-binding", action="store_true",
                    help="skip the second comparison with dt capped at 1e-4 h instead of 1e-6 h")
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--profile-steps", type=int, default=200)
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------
def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def dist_init(backend):
    import datetime
    import torch.distributed as dist
    rank, world, _ = dist_env()
    if world > 1 and not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


def reduce_max(x, device, world):
    """Max of a float over ranks (identity for one rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.rows = []
        self.t0 = self.t1 = None

    def start(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=timestamp," + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)

    def mark(self, which):
        setattr(self, which, time.time())

    def stop(self):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [ln.strip().split(", ") for ln in self.f.read().splitlines() if ln.strip()]
        self.f.close()
        os.unlink(self.f.name)
        out = []
        for r in rows:
            if len(r) < 10:
                continue
            try:
                out.append(dict(sm=float(r[2]), sm_max=float(r[3]), power=float(r[4]),
                                hw=r[6], hw_thermal=r[7], sw_thermal=r[8], sw_power=r[9]))
            except ValueError:
                continue
        self.rows = out
        return self.summary()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        reasons = set()
        for r in self.rows:
            for k, name in (("hw", "hw_slowdown"), ("hw_thermal", "hw_thermal_slowdown"),
                            ("sw_thermal", "sw_thermal_slowdown"), ("sw_power", "sw_power_cap")):
                if r[k].strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in self.rows),
                "sm_max_mhz": max(r["sm_max"] for r in self.rows), "reasons": sorted(reasons),
                "samples": len(self.rows)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def workload(n, seed, lib=None):
    """The seeded 100k-cell state.  `lib`: the oracle's build of the generator, so that the
    reference arm draws the same state without loading the product library."""
    from abm_b200 import workloads
    radius = 300.0 * (n / 100000.0) ** 0.5
    return workloads.biofilm_3d(n=n, seed=seed, disk_radius=radius, p_contact=P_CONTACT, lib=lib)


def oracle_module():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ref
    return oracle_ref


VARIANTS = {"plain": dict(precision=0, controller=0), "chosen": dict(precision=1, controller=1)}


def sim_params(args, n, variant="plain"):
    d = dict(cap_cells=n, integration_mode=args.tableau, pair_lanes=args.lanes, pair_tile=args.tile,
             pair_blocks_per_sm=args.bpsm, pair_sum=args.pair_sum,
             max_stepsize=1e-6, max_error_allowed=1e-8, iter_update_neighbors=100)
    d.update(VARIANTS[variant])
    return d


def stepsize_weights(path=None):
    """The shipped step-size network (trained on the GPU from reference-controller
    logs, abm_b200/stepsize.py), or the weights at `path`; trained here on the spot
    if the shipped file is missing."""
    from abm_b200 import stepsize
    if path:
        return stepsize.load(path), "weights from %s" % os.path.basename(path)
    if os.path.exists(stepsize.WEIGHTS_FILE):
        return stepsize.load(), "shipped weights (%s)" % os.path.basename(stepsize.WEIGHTS_FILE)
    w, info = stepsize.train_protocol(stepsize.default_runs(), n_iters=1500, epochs=150)
    return w, "trained at start on the GPU: %s" % json.dumps(info)


def config(args, info, extra=None):
    c = {"workload": "3d_mechanics_n%d_disk300um_z10um_%s_tol1e-8" %
                     (args.n, {1: "HE21", 2: "BS32", 3: "RKF45", 4: "DP54"}[args.tableau]),
         "cells": args.n, "tableau": {1: "HE21", 2: "BS32", 3: "RKF45", 4: "DP54"}[args.tableau],
         "rk_tol": 1e-8, "max_stepsize_h": 1e-6, "iter_update_neighbors": 100,
         "adhesion": "JKR isotropic gamma=100", "variant": args.variant,
         "precision": "mixed (FP32 segment distance + pair force)" if args.variant == "chosen" else "fp64",
         "controller": "learned (network proposal, error test)" if args.variant == "chosen" else "reference",
         "mean_contacts_per_cell": round(info["mean_contacts_per_cell"], 3),
         "l2": "flushed between timed steps (256 MB write)", "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


# algorithmic (unique) bytes per launch of each kernel, per cell
def pair_force_bytes(n, n_dir):
    # own geometry record 64 B + row_ptr 8 B + its neighbor indices 4 B each + dE/dq write 48 B
    return n * (64 + 8 + 48) + 4 * n_dir


def attempt_bytes(n, final):
    # geometry 64 + stored velocity 48 + physical record 64 + pair force 48 read;
    # the accepted attempt also writes geometry 64 + velocity 48 + length 8
    return n * (224 + (120 if final else 0))


def load_traffic():
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU baseline: the oracle run the way the reference runs
# ---------------------------------------------------------------------------
def oracle_for(cells, args, n_threads):
    """The oracle on the benchmark state, with its O(n^2) getCellNeighbors done (timed)."""
    import abm_b200                                  # parameter structs only: no library load
    orc = oracle_module()
    _, pd = abm_b200.make_params(**{k: v for k, v in sim_params(args, args.n).items()
                                   if k not in ("cap_cells", "precision", "pair_lanes", "controller")})
    o = orc.Oracle(pd, jkr=orc.jkr_table(0.8, 0.5, 3900.0, 100.0, 100), n_threads=n_threads)
    o.set_cells(cells)
    t0 = time.perf_counter()
    o.loop_init()                                  # O(n^2) getCellNeighbors
    return o, pd, time.perf_counter() - t0


def cpu_reference_rate(o, pd, t_build, args, steps):
    t0 = time.perf_counter()
    o.iterate(steps, 0, 0)                         # pair forces recomputed per stage
    t_steps = time.perf_counter() - t0
    k = pd["iter_update_neighbors"]
    t_amort = t_steps + t_build * steps / k
    value = args.n * steps / t_amort
    sample = ("%d accepted steps at n=%d (%.2f s) + one O(n^2) neighbor build (%.2f s) charged at the "
              "reference cadence of one rebuild per %d steps" % (steps, args.n, t_steps, t_build, k))
    return value, sample, dict(t_build_s=t_build, t_steps_s=t_steps)


def cpu_optimized_rate(cells, args, n_threads, steps):
    """The "optimized CPU" figure, for context beside the reference-faithful run: the
    oracle with a cell-list neighbor build, the stage-invariant pair forces evaluated once
    per attempt with OpenMP over the pairs, and OpenMP on every per-cell loop.  Same state,
    tableau, tolerance and controller; the build is charged at one per 100 steps as for the
    faithful run.  Not the reference's procedure, and not the baseline of any ratio."""
    import abm_b200                                  # parameter structs only: no library load
    orc = oracle_module()
    _, pd = abm_b200.make_params(**{k: v for k, v in sim_params(args, args.n).items()
                                   if k not in ("cap_cells", "precision", "pair_lanes", "controller")})
    o = orc.Oracle(pd, jkr=orc.jkr_table(0.8, 0.5, 3900.0, 100.0, 100), n_threads=n_threads,
                   n_start_multithread=1, cpu_optimized=True)
    o.set_cells(cells)
    t0 = time.perf_counter()
    o.loop_init()                                  # cell-list getCellNeighbors
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    o.iterate(steps, 0, 1)                         # pair forces once per attempt
    t_steps = time.perf_counter() - t0
    k = pd["iter_update_neighbors"]
    value = len(cells) * steps / (t_steps + t_build * steps / k)
    return {"value": value, "unit": UNIT, "cores": n_threads,
            "sample": ("%d accepted steps at n=%d (%.2f s) + one cell-list neighbor build (%.3f s) charged at "
                       "one rebuild per %d steps" % (steps, len(cells), t_steps, t_build, k)),
            "procedures": "cell-list neighbor build; pair forces once per attempt, OpenMP over the pairs; "
                          "OpenMP on the per-cell loops"}


def cpu_info():
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return os.cpu_count() or 1, model


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------
def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return                                     # rank 0 alone times the host reference
    # the oracle's build of the generator: this arm loads no product library
    cells, info = workload(args.n, SEED, lib=oracle_module().LIB)
    cores, model = cpu_info()
    # each reference step is one accepted iteration at n = 100k (~0.1-0.5 s on the host);
    # the run is bounded to about two minutes of CPU work
    steps = max(1, min(args.steps, 60))
    o, pd, t_build = oracle_for(cells, args, cores)
    value, sample, extra = cpu_reference_rate(o, pd, t_build, args, steps)
    ms = 1000.0 * args.n / value
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "warmup": 0, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded biofilm state)",
            "impl": "reference",
            "config": config(args, info, {"cpu_model": model, "requested_steps": args.steps,
                                          "variant": "reference CPU path", "precision": "fp64",
                                          "controller": "reference"}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def make_sim(args, variant, cells, weights, **over):
    import abm_b200
    sim = abm_b200.Simulation(**dict(sim_params(args, args.n, variant), **over))
    sim.upload_cells(cells)
    if VARIANTS[variant]["controller"] == 1:
        sim.set_stepsize_weights(weights)
    pairs = sim.get_cell_neighbors()
    return sim, pairs


def time_variant(sim, args, stream, flush, world, device, local):
    """W untimed iterations, then K timed ones (CUDA events on the context stream,
    L2 flushed before each), max over ranks."""
    import torch
    sim.iterate(max(args.warmup, 0), stats=False)
    sim.synchronize()
    s0 = sim.stats()
    sampler = ClockSampler(local)
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            sim.iterate(1, stats=False)
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    sim.synchronize()
    ms_total = reduce_max(sum(a.elapsed_time(b) for a, b in ev), device, world)
    s1 = sim.stats()
    d = {k: s1[k] - s0[k] for k in ("iterations", "attempts", "retries", "rejected", "rebuilds")}
    d.update(ms_total=ms_total, clocks=clocks, t_sim_h=s1["t"] - s0["t"])
    return d


def kernel_groups(sim, args, variant):
    """Per-kernel-group event timing (the iteration without the graph) and algorithmic bytes."""
    prof = sim.profile_iterations(max(1, min(args.profile_steps, args.steps)))
    n_dir = 2 * sim.stats()["n_pairs"]
    pf_ms = prof["pair_force_ms"] / prof["pair_force_launches"]
    at_ms = prof["attempt_ms"] / prof["iterations"]
    if VARIANTS[variant]["controller"] == 1:
        # the pair pass (its last block makes the network's proposal), then one RK
        # attempt that tests the proposal and advances the state in place
        pf_name = "k_pair_pass(+proposal)"
        at_name, at_bytes = "k_attempt(proposal)", attempt_bytes(args.n, True)
    else:
        pf_name = "k_pair_pass"
        at_name, at_bytes = "k_attempt(trial+final)", attempt_bytes(args.n, False) + attempt_bytes(args.n, True)
    kernels = {pf_name: (pair_force_bytes(args.n, n_dir), pf_ms), at_name: (at_bytes, at_ms)}
    return kernels, prof["rebuild_ms"] / max(prof["rebuild_launches"], 1)


def roofline(kernels, rebuild_ms):
    peak, peak_kind = measured_peak_hbm()
    traffic = load_traffic()
    dom = max(kernels, key=lambda k: kernels[k][1])
    b, ms = kernels[dom]
    achieved = b / (ms / 1000.0) / 1e9
    tr = traffic.get(dom, {}).get("bytes_per_launch")
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": tr, "kernel": dom,
            "algorithmic_bytes_per_launch": b, "ms_per_launch": ms, "peak_source": peak_kind,
            "other_kernels": {k: {"ms_per_launch": v[1], "algorithmic_bytes_per_launch": v[0],
                                  "achieved_gbs": v[0] / (v[1] / 1000.0) / 1e9}
                              for k, v in kernels.items() if k != dom},
            "rebuild_ms_per_rebuild": rebuild_ms}


def launches(variant, t, max_tries=3):
    # per iteration: the pair pass, then the attempts.  Reference controller: the trial,
    # its retries (WHILE node) and the final attempt.  Learned controller: the pair
    # pass also makes the proposal; the trial closes a passing step, and only a failed
    # proposal runs the IF node's max_tries retry launches and the final attempt.
    # 18 kernels per neighbor rebuild.
    learned = VARIANTS[variant]["controller"] == 1
    if learned:
        return t["iterations"] * 2 + t["rejected"] * (max_tries + 1) + 18 * t["rebuilds"]
    return t["iterations"] * 3 + t["retries"] + 18 * t["rebuilds"]


def relerr(a, b):
    """(max, rms) over columns of normwise relative errors |a - b| / |b|."""
    import numpy as np
    a, b = np.asarray(a), np.asarray(b)
    mx, rms = 0.0, 0.0
    for c in range(b.shape[1]):
        sb = np.abs(b[:, c]).max()
        if sb == 0:
            continue
        mx = max(mx, float(np.abs(a[:, c] - b[:, c]).max() / sb))
        rms = max(rms, float(np.sqrt(np.mean((a[:, c] - b[:, c]) ** 2) / np.mean(b[:, c] ** 2))))
    return {"max_rel": mx, "rms_rel": rms}


def gpu_step_outputs(args, cells, dt=1e-6):
    """Pair forces dE/dq, velocities, and one RK attempt at dt (new cells and the
    controller's scaled error norm E) of both precisions on the benchmark state."""
    import abm_b200
    out = {}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        sim = abm_b200.Simulation(cap_cells=args.n, integration_mode=args.tableau, precision=prec,
                                  max_stepsize=1e-6, max_error_allowed=1e-8)
        sim.upload_cells(cells)
        sim.get_cell_neighbors()
        f = sim.cell_cell_forces()
        v = sim.get_velocities()
        c1, _, e = sim.step_runge_kutta_adaptive(dt)
        out[name] = dict(forces=f, velocities=v, cells=c1, E=e)
        sim.close()
    return out


def rk_units(c_a, c_b, cells, tol=1e-8):
    """The error test's own units (simulation.hpp:1697-1705): max over cells and the six
    coordinates of |y1_a - y1_b| / (tol (1 + |y0|))."""
    import numpy as np
    y0 = cells[:, 1:7]
    return float((np.abs(c_a[:, 1:7] - c_b[:, 1:7]) / (tol * (1 + np.abs(y0)))).max())


def step_errors(gpu, ref, cells, against, dt=1e-6):
    """Per-step error of both GPU precisions against `ref` (the CPU oracle, or the FP64
    path when the oracle leg is skipped): forces and velocities as normwise relative
    errors, and the RK step in the error test's units beside the step's own scaled
    error norm E (what the error test compares with 1)."""
    out = {"against": against, "dt_h": dt}
    for name in ("mixed", "fp64"):
        g = gpu[name]
        out[name] = {"pair_forces": relerr(g["forces"], ref["forces"]),
                     "velocities": relerr(g["velocities"], ref["velocities"]),
                     "step_in_rk_units": rk_units(g["cells"], ref["cells"], cells),
                     "scaled_error_norm": g["E"]}
    out["reference_scaled_error_norm"] = ref["E"]
    return out


def oracle_step_outputs(o, dt=1e-6):
    c1, _, e = o.rk_attempt(dt)
    return dict(forces=o.cell_cell_forces(), velocities=o.get_velocities(), cells=c1, E=e)


def step_byte_model(P, E, s, K=100):
    """Algorithmic bytes per accepted cell-step of the FP64 plain path, B_step(s, P, E, K):
    pair refresh and force [8P + 56 + 48], E evaluations of B_eval(s) = 232 s + 24 s (s - 1)
    + 144 + 48 s, growth 24, and the cell list and pair build amortised over K."""
    b_eval = 232 * s + 24 * s * (s - 1) + 144 + 48 * s
    return (8 * P + 56 + 48) + E * b_eval + 24 + (56 + 4 + 16 + 8 * P) / K


STAGES = {1: 2, 2: 4, 3: 6, 4: 7}


def rebuild_cost(sim, stream, flush, steady_ms):
    """Device time a periodic neighbor rebuild adds to the loop: the iteration that
    launches it and the one after (whose pair pass screens every pair again), each timed
    like a step (L2 flushed before it), minus two steady steps."""
    import torch
    K = sim.params.iter_update_neighbors
    it = sim.clock()[2]
    sim.iterate((K - 1 - it % K) % K, stats=False)      # up to the iteration that launches it
    r0 = sim.stats()["rebuilds"]
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(2)]
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for a, b in ev:
            flush.zero_()
            a.record(stream)
            sim.iterate(1, stats=False)
            b.record(stream)
    torch.cuda.synchronize()
    assert sim.stats()["rebuilds"] == r0 + 1, "the timed pair of iterations must hold one rebuild"
    ms = sum(a.elapsed_time(b) for a, b in ev)
    return max(0.0, ms - 2 * steady_ms), ms


def time_binding(args, variant, cells, weights, flush, world, device, local, rebuild_extra_ms):
    """The same variant with dt free to grow to 1e-4 h, where the error test, not the cap,
    sets the step: W + 10 untimed iterations (dt climbs from 1e-6 h by at most 10x per
    step), then `steps` timed ones as in time_variant."""
    import torch
    a = argparse.Namespace(**vars(args))
    a.warmup = args.warmup + 10
    sim, _ = make_sim(args, variant, cells, weights, max_stepsize=BINDING_MAX_DT)
    stream = torch.cuda.ExternalStream(sim.stream, device=device)
    t = time_variant(sim, a, stream, flush, world, device, local)
    sim.close()
    K = 100
    charge = max(0.0, args.steps / K - t["rebuilds"]) * rebuild_extra_ms
    ms = t["ms_total"] + charge
    return {"value": world * args.n * args.steps / (ms / 1000.0), "ms_per_step": ms / args.steps,
            "rk_evals_per_step": round(t["attempts"] / max(t["iterations"], 1), 3),
            "rejected_first_attempts": t["rejected"], "retries": t["retries"],
            "simulated_h_in_timed_region": t["t_sim_h"], "simulated_h_per_s": t["t_sim_h"] / (ms / 1000.0),
            "rebuild_charge_ms": charge,
            "clocks": {k: t["clocks"][k] for k in ("sm_mhz", "sm_max_mhz", "reasons")}}


def run_b200(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        dist_init("nccl")
    cells, info = workload(args.n, SEED + rank)
    weights, weights_note = stepsize_weights(args.weights)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=device)

    head = args.variant
    other = None if args.only else ("plain" if head == "chosen" else "chosen")
    results = {}
    for variant in [v for v in (other, head) if v]:
        sim, pairs = make_sim(args, variant, cells, weights)
        stream = torch.cuda.ExternalStream(sim.stream, device=device)
        t = time_variant(sim, args, stream, flush, world, device, local)
        t["pairs"] = pairs
        t["kernels"], _ = kernel_groups(sim, args, variant)
        # the periodic rebuild (one per iter_update_neighbors = 100 iterations) at its share
        # of the timed steps, when the timed region held fewer than its share
        steady = t["ms_total"] / args.steps
        t["rebuild_extra_ms"], t["rebuild_pair_ms"] = rebuild_cost(sim, stream, flush, steady)
        t["rebuild_extra_ms"] = reduce_max(t["rebuild_extra_ms"], device, world)
        t["rebuild_charge_ms"] = max(0.0, args.steps / 100 - t["rebuilds"]) * t["rebuild_extra_ms"]
        t["ms_charged"] = t["ms_total"] + t["rebuild_charge_ms"]
        t["value"] = world * args.n * args.steps / (t["ms_charged"] / 1000.0)
        if variant == head:
            # e2e through the C ABI with pinned host buffers
            ncols = cells.shape[1]
            host = torch.empty((ncols, args.n), dtype=torch.float64, pin_memory=True)
            host.numpy()[:] = sim.download_cells().T
            ptr = host.data_ptr()
            e2e_steps = max(1, min(args.steps, 200))
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            barrier(world)
            e0.record(stream)
            for _ in range(e2e_steps):
                sim.upload_cells_raw(ptr, args.n, ncols, args.n)
                sim.iterate(1, stats=False)
                sim.download_cells_raw(ptr, args.n)
            e1.record(stream)
            torch.cuda.synchronize()
            e2e_ms = reduce_max(e0.elapsed_time(e1), device, world)
            nbytes = args.n * ncols * 8
            t["e2e"] = {"value": world * args.n * e2e_steps / (e2e_ms / 1000.0), "unit": UNIT,
                        "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "steps": e2e_steps}
        sim.close()
        results[variant] = t

    h = results[head]
    P = h["pairs"] / args.n
    E = h["attempts"] / max(h["iterations"], 1)
    b_step = step_byte_model(P, E, STAGES[args.tableau])
    roof = roofline(h["kernels"], h["rebuild_extra_ms"])
    peak = roof["peak"]
    roof["b_step_model"] = {"bytes_per_cell_step": b_step, "pairs_per_cell": P, "rk_evals_per_step": E,
                            "achieved": b_step * h["value"] / world / 1e9,
                            "frac": b_step * h["value"] / world / 1e9 / peak, "unit": "GB/s",
                            "note": "whole step, FP64 element widths, against the same peak"}
    line = {"metric": METRIC, "value": h["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": h["ms_charged"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32" if head == "chosen" else "f64",
            "data": "synthetic (seeded biofilm state, p_contact=%g)" % P_CONTACT,
            "config": config(args, info, {"pairs_per_cell": round(P, 3),
                                          "rk_evals_per_step": round(E, 3),
                                          "rejected_first_attempts": h["rejected"],
                                          "rebuilds_in_timed_region": h["rebuilds"],
                                          "rebuild_charge_ms": h["rebuild_charge_ms"],
                                          "simulated_h_in_timed_region": h["t_sim_h"],
                                          "stepsize_network": weights_note if head == "chosen" else None}),
            "e2e": h["e2e"], "gpu_launches": launches(head, h),
            "roofline": roof,
            "clocks": {k: h["clocks"][k] for k in ("sm_mhz", "sm_max_mhz", "reasons")}}
    if other:
        o = results[other]
        line[other] = {"value": o["value"], "ms_per_step": o["ms_charged"] / args.steps,
                       "rk_evals_per_step": round(o["attempts"] / max(o["iterations"], 1), 3),
                       "rejected_first_attempts": o["rejected"], "simulated_h_in_timed_region": o["t_sim_h"],
                       "rebuild_charge_ms": o["rebuild_charge_ms"],
                       "kernels_ms_per_launch": {k: v[1] for k, v in o["kernels"].items()},
                       "clocks": {k: o["clocks"][k] for k in ("sm_mhz", "sm_max_mhz", "reasons")}}
        chosen, plain = results["chosen"], results["plain"]
        line["chosen_over_plain"] = {"accepted_cell_steps": chosen["value"] / plain["value"],
                                     "simulated_time_per_s": (chosen["t_sim_h"] / chosen["ms_charged"]) /
                                                             (plain["t_sim_h"] / plain["ms_charged"])}
        if not args.no_binding:
            bind = {v: time_binding(args, v, cells, weights, flush, world, device, local,
                                    results[v]["rebuild_extra_ms"]) for v in ("plain", "chosen")}
            bind["max_stepsize_h"] = BINDING_MAX_DT
            bind["chosen_over_plain"] = {
                "accepted_cell_steps": bind["chosen"]["value"] / bind["plain"]["value"],
                "simulated_time_per_s": bind["chosen"]["simulated_h_per_s"] / bind["plain"]["simulated_h_per_s"]}
            line["error_bound_dt"] = bind
    if rank == 0 and world == 1 and "chosen" in results:
        gpu = gpu_step_outputs(args, cells)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores, model = cpu_info()
        orc_obj, pd, t_build = oracle_for(cells, args, cores)
        if "chosen" in results:
            line["mixed_precision_error"] = step_errors(gpu, oracle_step_outputs(orc_obj), cells,
                                                        "CPU oracle (FP64 restatement of the reference)")
        v, sample, extra = cpu_reference_rate(orc_obj, pd, t_build, args, args.cpu_steps)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": sample + " on " + model}
        del orc_obj
        try:
            line["cpu_optimized"] = cpu_optimized_rate(cells, args, cores, 2 * args.cpu_steps)
        except Exception as e:                     # a context figure: never costs the line
            line["cpu_optimized"] = {"error": "%s: %s" % (type(e).__name__, e)}
    elif rank == 0 and world == 1 and "chosen" in results:
        line["mixed_precision_error"] = step_errors(gpu, gpu["fp64"], cells,
                                                    "FP64 path of this library (the oracle leg was skipped)")
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_replicates(args):
    """Batched 2-D replicates: args.replicates colonies with log-uniform target sizes in
    [500, 50000], each grown from one founder cell with its own seed (or, with
    --replicate-start near-target, from a seeded colony at 90 % of its target), with
    config-0 growth and division (BS32, tol 1e-8) until its target; one graph launch per
    iteration advances all of them.  The screened pair pass's shape per size decade
    comes from the autotuner.  W + K iterations are run; the line reports the K timed
    ones, whatever sizes the colonies have reached by then."""
    import torch
    from abm_b200 import replicates
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        dist_init("nccl")
    targets = replicates.target_sizes(args.replicates, 500, 50000, seed=rank)
    tiles = replicates.tiles_by_bucket(targets, replicates.CONFIG0)
    founders = args.replicate_start == "founder"
    bt, sims = replicates.make_batch(targets, seed=1000 * rank + 1, start_fraction=0.9, tiles=tiles,
                                     founders=founders)
    bt.iterate(max(args.warmup, 0))
    bt.synchronize()
    s0 = [s.stats() for s in sims]
    stream = torch.cuda.ExternalStream(bt.stream, device=device)
    sampler = ClockSampler(local)
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    bt.iterate(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    bt.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms = reduce_max(e0.elapsed_time(e1), device, world)
    s1 = [s.stats() for s in sims]
    d = {k: sum(b[k] - a[k] for a, b in zip(s0, s1)) for k in ("cell_steps", "iterations", "attempts",
                                                                "rejected", "retries", "divisions")}
    cells_now = sum(s.num_cells() for s in sims)
    halted = sum(1 for s, t in zip(sims, targets) if s.num_cells() >= t)
    value = world * d["cell_steps"] / (ms / 1000.0)
    line = {"metric": "accepted cell-steps/s, batched 2D replicates", "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded 2-D colonies)",
            "config": {"workload": "2d_replicates_%d_loguniform500-50000_BS32_tol1e-8_from_%s" %
                                   (args.replicates, "founder" if founders else "90pct_of_target"),
                       "replicates": args.replicates, "cells_at_end": cells_now,
                       "target_cells_total": int(targets.sum()), "replicates_at_target": halted,
                       "rejected_step_fraction": d["rejected"] / max(d["iterations"], 1),
                       "rk_evals_per_step": d["attempts"] / max(d["iterations"], 1),
                       "divisions": d["divisions"], "l2": "state larger than L2 (no flush needed)",
                       "pair_tile_by_size_decade": {str(10 ** b): list(v[0]) for b, v in tiles.items()},
                       "parallelism": "replicas"},
            "gpu_launches": None,
            "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    bt.close()
    for s in sims:
        s.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def grow_arm(args, variant, weights, device, seed):
    """One arm of the growth run: founder -> args.growth_target cells on the device."""
    import torch
    import abm_b200
    from abm_b200 import stepsize, workloads
    kw = dict(stepsize.GROWTH_KW, daughter_length_std=0.01)
    target = args.growth_target
    sim = abm_b200.Simulation(cap_cells=int(1.05 * target) + 4096, integration_mode=args.tableau,
                              max_stepsize=args.growth_max_dt, max_error_allowed=1e-8, iter_update_neighbors=100,
                              rng_seed=seed, **dict(kw, **VARIANTS[variant]))
    try:
        sim.upload_cells(workloads.founder_3d())
        if VARIANTS[variant]["controller"] == 1:
            sim.set_stepsize_weights(weights)
        sim.set_parents([-1])
        sim.set_clock(0.0, 1e-6, 0)          # dt0 = 1e-6 h
        sim.set_cell_limit(target)
        sim.get_cell_neighbors()
        stream = torch.cuda.ExternalStream(sim.stream, device=device)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ms, chunk, error, n = 0.0, 512, None, 1
        st = dict.fromkeys(("iterations", "attempts", "rejected", "retries", "divisions", "t", "cell_steps"), 0)
        while True:
            try:
                st = sim.iterate(chunk)          # raises on a device-side error status
            except RuntimeError as e:
                error = str(e)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            n = sim.num_cells()
            if error or n >= target or ms > 1000.0 * args.growth_max_seconds:
                break
    finally:
        sim.close()
    return {"cells": n, "reached_target": n >= target, "error": error, "device_s": ms / 1000.0,
            "accepted_steps": st["iterations"], "rk_evals": st["attempts"],
            "rk_evals_per_step": st["attempts"] / max(st["iterations"], 1),
            "rejected_first_attempts": st["rejected"], "retries": st["retries"],
            "divisions": st["divisions"], "simulated_h": st["t"], "cell_steps": st["cell_steps"],
            "accepted_cell_steps_per_s": st["cell_steps"] / max(ms / 1000.0, 1e-9)}


def run_growth(args):
    """3-D growth from one founder cell to args.growth_target cells: growth rates
    ~ N(1.5, 0.1^2)/h, division at Ldiv = 2 L0 + 2R = 5.6 um into daughters split at a
    fraction ~ N(0.5, 0.01^2), Heun-Euler 2(1), RK tolerance 1e-8, dt0 = 1e-6 h, dt capped
    at args.growth_max_dt; plain (FP64, reference controller) then chosen (mixed
    precision, learned step size).  Each arm's device time runs from the founder to
    the target (CUDA events on the context stream); the colony stops on the device when
    it reaches the target."""
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        dist_init("nccl")
    weights, weights_desc = stepsize_weights(args.weights)
    sampler = ClockSampler(local)
    sampler.start()
    barrier(world)
    arms = {v: grow_arm(args, v, weights, device, seed=7 + rank) for v in args.growth_arms.split(",")}
    clocks = sampler.stop()
    ms = {v: reduce_max(1000.0 * a["device_s"], device, world) for v, a in arms.items()}
    ch = arms.get("chosen") or arms[next(iter(arms))]
    ms.setdefault("chosen", ms[next(iter(ms))])
    value = world * ch["cell_steps"] / (ms["chosen"] / 1000.0)
    line = {"metric": "3D growth founder -> %d cells: accepted cell-steps/s" % args.growth_target,
            "value": value, "unit": UNIT, "n_gpus": world, "steps": ch["accepted_steps"], "warmup": 0,
            "ms_per_step": ms["chosen"] / max(ch["accepted_steps"], 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic (one founder cell)",
            "config": {"workload": "3d_growth_founder_to_%d_HE21_tol1e-8_maxdt%g" % (args.growth_target,
                                                                                   args.growth_max_dt),
                       "variant": "chosen", "parallelism": "replicas", "stepsize_network": weights_desc,
                       "l2": "state larger than L2 after ~30k cells (no flush)"},
            "arms": arms,
            "chosen_over_plain": ({"device_time": ms["plain"] / max(ms["chosen"], 1e-9),
                                   "rk_evals": arms["plain"]["rk_evals"] / max(ch["rk_evals"], 1)}
                                  if "plain" in arms and "chosen" in arms else None),
            "gpu_launches": None,
            "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "replicates":
        run_replicates(args)
    elif args.workload == "growth":
        run_growth(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
