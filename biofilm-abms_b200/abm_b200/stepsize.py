"""Learned step-size controller: data, initialisation and training.

The network (32 features -> 64 -> 64 -> 1, ReLU) proposes ln(dt / dt_prev) for the
next RK step.  Training pairs come from the feature log a context writes while
the reference controller (simulation.hpp:1688-1769) runs: for every iteration
the features seen before its first attempt, and the largest step the embedded
error model accepts, dt_max = dt_first * E^(-1/(q+1)) with E the first attempt's
scaled error and q the tableau's error order.  The loop adds the network output
to the error-model baseline b = ln 0.9 - ln(E_last)/(q+1) of the last accepted
step, so the network's target is clamp(ln(safety dt_max / dt_prev), ln 0.2, ln 10) - b.

Training runs on the GPU (abm_mlp_train: BF16 tensor-core forward/backward,
FP32 Adam).  In the loop the proposal is one RK attempt that is accepted as is
when its error passes, and the reference rule takes over from that attempt
when it does not, so the error test decides every accepted step.
"""
import os

import numpy as np

from . import MLP_FEATURES, MLP_HIDDEN, MLP_NPARAM, mlp_train

LN_MIN, LN_MAX = float(np.log(0.2)), float(np.log(10.0))
WEIGHTS_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "stepsize_mlp.npz")


def training_pairs(rows, safety=0.9):
    """(X, T) from logged rows (n x 40): X = features, T = the network's share of
    the target, clamp(ln(safety dt_max / dt_prev), ln 0.2, ln 10) - b, where b is the
    error-model baseline the loop adds to the network output (column 36)."""
    rows = np.asarray(rows, dtype=np.float32)
    X = np.ascontiguousarray(rows[:, :MLP_FEATURES])
    T = rows[:, 33].astype(np.float64) + rows[:, 32] + np.log(safety)
    T = np.clip(T, LN_MIN, LN_MAX) - rows[:, 36]
    return X, T.astype(np.float32)


def init_weights(seed=0, out_bias=0.0):
    """He-normal hidden layers, small output layer, zero biases except the output's."""
    rng = np.random.default_rng(seed)
    w = np.zeros(MLP_NPARAM, dtype=np.float32)
    o = 0
    w[o:o + MLP_HIDDEN * MLP_FEATURES] = rng.normal(0, np.sqrt(2.0 / MLP_FEATURES), MLP_HIDDEN * MLP_FEATURES)
    o += MLP_HIDDEN * MLP_FEATURES + MLP_HIDDEN
    w[o:o + MLP_HIDDEN * MLP_HIDDEN] = rng.normal(0, np.sqrt(2.0 / MLP_HIDDEN), MLP_HIDDEN * MLP_HIDDEN)
    o += MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN
    w[o:o + MLP_HIDDEN] = rng.normal(0, 0.1 / np.sqrt(MLP_HIDDEN), MLP_HIDDEN)
    w[-1] = out_bias
    return w


def train(rows, epochs=300, lr=1e-3, seed=0, safety=0.9):
    """Train on logged rows with the GPU kernels; returns (weights, loss per epoch)."""
    X, T = training_pairs(rows, safety)
    w0 = init_weights(seed, out_bias=float(np.median(T)))
    return mlp_train(w0, X, T, epochs=epochs, lr=lr, seed=seed)


def save(weights, path=WEIGHTS_FILE, **meta):
    np.savez(path, weights=np.asarray(weights, np.float32), **meta)


def load(path=WEIGHTS_FILE):
    with np.load(path) as f:
        return f["weights"].astype(np.float32)


# ---------------------------------------------------------------------------
# Logged runs and the training protocol
# ---------------------------------------------------------------------------
GROWTH_KW = dict(growth_mean=1.5, growth_std=0.1, daughter_length_std=0.05, daughter_angle_xy_bound=0.3,
                 daughter_angle_z_bound=0.1)


def growing_colony(n, seed, growth_mean=1.5, growth_std=0.1, lmax=5.5):
    """Seeded 3-D colony at the 100k-benchmark density with per-cell growth rates
    ~ N(growth_mean, growth_std^2) and lengths up to just below Ldiv, so that cells
    divide during a run."""
    from . import workloads
    cells, _ = workloads.biofilm_3d(n=n, seed=seed, disk_radius=300.0 * np.sqrt(n / 1e5), p_contact=0.9,
                                    lmax=lmax)
    rng = np.random.default_rng(seed + 1000)
    cells[:, 16] = rng.normal(growth_mean, growth_std, n)
    return cells


def founder_colonies(sizes, seed=7, max_stepsize=1e-4, max_iters=20_000_000):
    """Grow a 3-D colony from one founder cell (the 3-D driver's start, growth
    ~ N(1.5, 0.1^2)/h, daughters split at ~ N(0.5, 0.01^2)) with the reference
    controller and return a copy of its cells as it reaches each of `sizes`."""
    from . import Simulation, workloads
    kw = dict(GROWTH_KW, daughter_length_std=0.01)
    sizes = sorted(sizes)
    sim = Simulation(cap_cells=int(1.05 * sizes[-1]) + 4096, max_stepsize=max_stepsize, rng_seed=seed, **kw)
    out = []
    try:
        sim.upload_cells(workloads.founder_3d())
        sim.set_parents([-1])
        sim.set_clock(0.0, 1e-6, 0)
        sim.get_cell_neighbors()
        done = 0
        for target in sizes:
            sim.set_cell_limit(target)
            while sim.num_cells() < target and done < max_iters:
                sim.iterate(4096, stats=False)
                done += 4096
            out.append(sim.download_cells())
    finally:
        sim.close()
    return out


def logged_run(cells, n_iters, controller=0, weights=None, max_stepsize=1e-4, log_capacity=None, **params):
    """Run n_iters iterations from `cells` with the feature log on; returns (rows, stats)."""
    from . import Simulation
    n = cells.shape[0]
    cap = log_capacity or n_iters
    kw = dict(GROWTH_KW)
    kw.update(params)
    sim = Simulation(cap_cells=max(4 * n, 64), max_stepsize=max_stepsize, controller=controller,
                     stepsize_log_capacity=cap, **kw)
    try:
        sim.upload_cells(cells)
        if weights is not None:
            sim.set_stepsize_weights(weights)
        sim.set_clock(0.0, max_stepsize, 0)
        sim.get_cell_neighbors()
        st = sim.iterate(n_iters)
        rows = sim.stepsize_log()
    finally:
        sim.close()
    return rows, st


def train_protocol(runs, n_iters=3000, epochs=200, lr=1e-3, seed=0, safety=0.9, aggregate_rounds=1):
    """Train from reference-controller logs of `runs` (a list of (cells, params)),
    then `aggregate_rounds` times add the learned controller's own logs on the
    same states and retrain (data aggregation).  Returns (weights, info)."""
    rows = [logged_run(c, n_iters, controller=0, **p)[0] for c, p in runs]
    data = np.concatenate(rows)
    w, losses = train(data, epochs=epochs, lr=lr, seed=seed, safety=safety)
    info = {"rows_reference": int(len(data)), "loss_first": float(losses[0]), "loss_last": float(losses[-1])}
    for r in range(aggregate_rounds):
        own = [logged_run(c, n_iters, controller=1, weights=w, **p)[0] for c, p in runs]
        data = np.concatenate([data] + own)
        w, losses = train(data, epochs=epochs, lr=lr, seed=seed + 1 + r, safety=safety)
        info["rows_round%d" % (r + 1)] = int(len(data))
        info["loss_last_round%d" % (r + 1)] = float(losses[-1])
    return w, info


def default_runs(founders=False):
    """The logged runs behind the shipped weights: 3-D growth with division at
    three colony sizes (error-limited, max_stepsize 1e-4) and the static 100k-density
    state at max_stepsize 1e-6, each from its own seed.  founders adds compact
    colonies grown from one founder cell to 1,000 and 4,000 cells; weights trained
    with them performed the same on founder growth (30 % instead of 34 % rejected
    proposals, the same simulated time per second), so the shipped ones do without."""
    runs = []
    for n, seed in ((500, 11), (2000, 12), (8000, 13)):
        runs.append((growing_colony(n, seed), dict(max_stepsize=1e-4)))
    runs.append((growing_colony(20000, 14, growth_mean=0.0, growth_std=0.0, lmax=5.0), dict(max_stepsize=1e-6)))
    if founders:
        for cells in founder_colonies((1000, 4000)):
            runs.append((cells, dict(max_stepsize=1e-4, daughter_length_std=0.01)))
    return runs


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the step-size network on the GPU and save its weights")
    ap.add_argument("--out", default=WEIGHTS_FILE)
    ap.add_argument("--iters", type=int, default=3000)
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--founders", action="store_true", help="add the founder-grown colonies to the runs")
    a = ap.parse_args(argv)
    w, info = train_protocol(default_runs(founders=a.founders), n_iters=a.iters, epochs=a.epochs, seed=a.seed)
    save(w, a.out, info=json.dumps(info))
    print(json.dumps(info))


if __name__ == "__main__":
    main()
