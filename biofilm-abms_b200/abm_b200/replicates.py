"""Batched 2-D replicate biofilms (many independent colonies of uneven size
advanced together, each with its own seed, clock and adaptive step).

The 2-D driver (ABM-2d/ABM-2d-cpp/include/simulation.hpp:163-237) runs one colony
per job; here every replicate is a context of its own and a Batch advances all of
them with one CUDA graph launch per iteration.  The screened pair pass's tile and
grid shape are picked per replicate-size decade by the autotuner
(abm_autotune_pair_tile).
"""
import numpy as np

from . import DEFAULTS_2D, Batch, Simulation, autotune_pair_tile, workloads

# config-0 mechanics and growth: R 0.8, Hertz E0 3900, Ldiv 4.4, growth N(1.5, 0.1^2),
# daughter fraction N(0.5, 0.01^2), BS32 at tol 1e-8
CONFIG0 = dict(DEFAULTS_2D, R=0.8, Rcell=0.5, E0=3900.0, Ecell=3.9e6, Ldiv=4.4, neighbor_threshold=3.2,
               growth_mean=1.5, growth_std=0.1, daughter_length_std=0.01, daughter_angle_xy_bound=0.05,
               max_error_allowed=1e-8, min_error=1e-30, max_stepsize=1e-4, min_stepsize=1e-9,
               iter_update_neighbors=100)


def target_sizes(n_rep=256, lo=500, hi=50000, seed=0):
    """Log-uniform target sizes on [lo, hi] (seeded)."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n_rep)).astype(int)


def start_state(n, seed, growth_mean=1.5, growth_std=0.1, Ldiv=4.4):
    """A seeded colony of n cells at the 2-D benchmark density with per-cell growth
    rates ~ N(growth_mean, growth_std^2) and lengths up to just below Ldiv."""
    cells = workloads.biofilm_2d(n, seed=seed, lmin=1.4, lmax=Ldiv - 0.05)
    rng = np.random.default_rng(seed + 7919)
    cells[:, 12] = rng.normal(growth_mean, growth_std, n)
    return cells


def tiles_by_bucket(sizes, params, seed=0, launches=10):
    """Autotune the screened pair pass's (tile, blocks per SM) once per decade of replicate size."""
    buckets = sorted(set(int(np.floor(np.log10(max(s, 1)))) for s in sizes))
    out = {}
    for b in buckets:
        n = int(min(max(3 * 10 ** b, 200), 30000))
        best, times = autotune_pair_tile(start_state(n, seed + b), launches=launches, cap_cells=n,
                                         **{k: v for k, v in params.items() if k != "cap_cells"})
        out[b] = (best, times)
    return out


def make_batch(targets, seed=0, start_fraction=0.9, tiles=None, founders=False, **overrides):
    """Replicate r: a colony of start_fraction * targets[r] cells (or one founder cell)
    with seed seed + r, stopping at targets[r] cells.  Returns (Batch, [Simulation])."""
    params = dict(CONFIG0)
    params.update(overrides)
    sims = []
    for r, tgt in enumerate(targets):
        cells = workloads.founder_2d() if founders else start_state(max(1, int(start_fraction * tgt)), seed + r)
        p = dict(params)
        p["cap_cells"] = int(2 * tgt + 64)
        p["rng_seed"] = seed + r
        if tiles is not None:
            b = int(np.floor(np.log10(max(tgt, 1))))
            if b in tiles:
                p["pair_tile"], p["pair_blocks_per_sm"] = tiles[b][0]
        sim = Simulation(**p)
        sim.upload_cells(cells)
        sim.set_parents(-np.ones(cells.shape[0], dtype=np.int32))
        sim.set_clock(0.0, p["max_stepsize"], 0)
        sim.set_cell_limit(int(tgt))
        sim.get_cell_neighbors()
        sims.append(sim)
    return Batch(sims), sims
