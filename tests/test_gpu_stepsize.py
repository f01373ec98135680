"""Step-size network on the GPU: forward and gradient against the CPU
restatement (oracle/mlp_ref.py), training, the in-loop proposal, and the
learned controller's accepted step against the oracle's RK step."""
import numpy as np
import pytest

import abm_b200
from abm_b200 import stepsize, workloads
import mlp_ref
import oracle_ref as orc

pytestmark = pytest.mark.gpu

JKR = orc.jkr_table(0.8, 0.5, 3900.0, 100.0, 100)


def problem(n, seed):
    rng = np.random.default_rng(seed)
    w = stepsize.init_weights(seed, out_bias=0.2)
    w[mlp_ref.OFF_B1:mlp_ref.OFF_W2] = rng.normal(0, 0.1, 64)
    w[mlp_ref.OFF_B2:mlp_ref.OFF_W3] = rng.normal(0, 0.1, 64)
    X = rng.normal(0, 1, (n, 32)).astype(np.float32)
    T = (np.tanh(X[:, :4].sum(1) / 2) + 0.1 * X[:, 5]).astype(np.float32)
    return w, X, T


def test_mlp_forward_matches_cpu_restatement():
    w, X, _ = problem(1003, 1)                 # not a multiple of the 16-row tile
    y = abm_b200.mlp_forward(w, X)
    yo, _, _ = mlp_ref.forward(w, X)
    # same BF16 operands on both sides; FP32 vs FP64 accumulation can move a hidden
    # activation across a BF16 rounding boundary (one BF16 ulp, 2^-8 relative)
    assert np.abs(y - yo).max() <= 2e-3 * (1 + np.abs(yo).max())
    assert np.median(np.abs(y - yo)) <= 1e-5 * (1 + np.abs(yo).max())


def test_mlp_gradient_matches_cpu_restatement():
    w, X, T = problem(1003, 2)
    g, loss = abm_b200.mlp_grad(w, X, T)
    go, losso = mlp_ref.grad(w, X, T)
    assert abs(loss - losso) <= 1e-4 * losso
    assert np.linalg.norm(g - go) <= 2e-3 * np.linalg.norm(go)
    blocks = [(mlp_ref.OFF_W1, mlp_ref.OFF_B1), (mlp_ref.OFF_B1, mlp_ref.OFF_W2), (mlp_ref.OFF_W2, mlp_ref.OFF_B2),
              (mlp_ref.OFF_B2, mlp_ref.OFF_W3), (mlp_ref.OFF_W3, mlp_ref.OFF_B3), (mlp_ref.OFF_B3, mlp_ref.NPARAM)]
    for a, b in blocks:
        assert np.linalg.norm(g[a:b] - go[a:b]) <= 5e-3 * np.linalg.norm(go[a:b]) + 1e-7, (a, b)
    # and the rounded network's gradient is close to the exact FP64 gradient
    g64, _ = mlp_ref.grad_fp64(w, X, T)
    assert np.linalg.norm(g - g64) <= 3e-2 * np.linalg.norm(g64)


def test_mlp_training_reduces_the_loss():
    w, X, T = problem(4096, 3)
    _, loss0 = abm_b200.mlp_grad(w, X, T)
    w1, losses = abm_b200.mlp_train(w, X, T, epochs=60, lr=2e-3, seed=5)
    _, loss1 = abm_b200.mlp_grad(w1, X, T)
    assert loss1 < 0.1 * loss0, (loss0, loss1)
    assert losses[-1] < losses[0]
    # the gradient sums use FP32 atomics, so a second run differs in rounding only
    w2, _ = abm_b200.mlp_train(w, X, T, epochs=60, lr=2e-3, seed=5)
    _, loss2 = abm_b200.mlp_grad(w2, X, T)
    assert loss2 < 0.1 * loss0


def colony(n, seed, growth=1.5):
    cells, _ = workloads.biofilm_3d(n=n, seed=seed, disk_radius=300.0 * np.sqrt(n / 1e5), p_contact=0.9)
    cells[:, 16] = growth
    return cells


def test_in_loop_proposal_is_the_network_output():
    cells = colony(1500, 31, growth=0.0)
    sim = abm_b200.Simulation(cap_cells=1600, jkr_table=JKR, controller=1, stepsize_log_capacity=64,
                              max_stepsize=1.0, min_stepsize=1e-15)
    sim.upload_cells(cells)
    w = stepsize.init_weights(7, out_bias=float(np.log(0.7)))
    sim.set_stepsize_weights(w)
    np.testing.assert_array_equal(sim.stepsize_weights(), w)
    sim.set_clock(0.0, 1e-6, 0)
    sim.get_cell_neighbors()
    sim.iterate(6)
    rows = sim.stepsize_log()
    assert rows.shape == (6, abm_b200.MLP_LOG_COLS)
    y = abm_b200.mlp_forward(w, rows[:, :32])
    # baseline: the PI ratio b = ln 0.9 - (0.7 ln E_last - 0.4 ln E_prev)/(q+1), HE21: q = 1,
    # ln E = ln(10) 10 x features 12 and 13
    ln10 = np.float32(2.302585093) * np.float32(10.0)
    b = np.log(0.9) - 0.5 * (0.7 * ln10 * rows[:, 12] - 0.4 * ln10 * rows[:, 13])
    np.testing.assert_allclose(rows[:, 36], b, rtol=1e-5, atol=1e-5)
    r = np.clip(rows[:, 36].astype(np.float64) + y, np.log(0.2), np.log(10.0))
    np.testing.assert_allclose(rows[:, 33], r, atol=2e-6)
    sim.close()


def test_learned_step_equals_the_oracle_rk_step():
    """A proposal that passes the error test is committed as is: the state equals
    the oracle's RK step at the proposed dt followed by growth (growth.hpp:51-57)."""
    cells = colony(3000, 32, growth=1.5)
    cells[:, 13] = np.minimum(cells[:, 13], 4.0)
    cells[:, 14] = cells[:, 13] / 2
    sim = abm_b200.Simulation(cap_cells=3100, jkr_table=JKR, controller=1, max_stepsize=1e-4)
    sim.upload_cells(cells)
    w = np.zeros(abm_b200.MLP_NPARAM, dtype=np.float32)
    # first iteration: no history, E_last = 1, baseline ln 0.9; output ln(0.5/0.9)
    w[-1] = np.log(0.5) - np.log(0.9)
    sim.set_stepsize_weights(w)
    sim.set_clock(0.0, 1e-6, 0)
    sim.get_cell_neighbors()
    s = sim.iterate(1)
    assert s["attempts"] == 1 and s["rejected"] == 0 and s["iterations"] == 1
    t, dt, it = sim.clock()
    assert it == 1 and abs(t - 1e-6 * 0.5) <= 1e-6 * 1e-6
    got = sim.download_cells()
    o = orc.Oracle(sim.pdict, jkr=JKR)
    o.set_cells(cells)
    o.build_neighbors()
    co, _, mo = o.rk_attempt(t)
    assert mo <= 1.0
    for c in range(1, 13):                    # r, n, then the stored velocities
        scale = np.abs(co[:, c]).max()
        assert np.abs(got[:, c] - co[:, c]).max() <= 1e-10 * max(scale, 1e-300), c
    l = cells[:, 13]
    lg = l + cells[:, 16] * (4 * 0.8 / 3 + l) * t
    np.testing.assert_allclose(got[:, 13], lg, rtol=1e-14, atol=0)
    np.testing.assert_allclose(got[:, 14], lg / 2, rtol=1e-14, atol=0)
    sim.close()


def test_rejected_proposal_falls_back_to_the_reference_rule():
    """A proposal far too large fails the error test; the reference rule then
    retries from that attempt and re-runs the final step, as simulation.hpp:1688-1769."""
    cells = colony(2000, 33, growth=0.0)
    sim = abm_b200.Simulation(cap_cells=2100, jkr_table=JKR, controller=1, max_stepsize=1.0)
    sim.upload_cells(cells)
    w = np.zeros(abm_b200.MLP_NPARAM, dtype=np.float32)
    w[-1] = 50.0                              # always ask for the largest step (10x)
    sim.set_stepsize_weights(w)
    sim.set_clock(0.0, 1e-3, 0)
    sim.get_cell_neighbors()
    s = sim.iterate(3)
    assert s["iterations"] == 3
    assert s["rejected"] >= 1
    assert s["attempts"] > s["iterations"]      # fallback iterations take more than one attempt
    assert np.isfinite(sim.download_cells()).all()
    sim.close()


@pytest.mark.parametrize("mode,noise", [(1, False), (2, False), (1, True)])
def test_rejected_proposal_matches_the_oracle_reference_iteration(mode, noise):
    """A proposal that fails the error test is followed by the reference rule, which
    restarts from the copy of y0 the trial kept (l in the gamma slot, the stored
    velocities beside it): the iteration must end where the oracle's reference-controller
    iteration (simulation.hpp:1688-1769) ends when it starts at the proposed dt -- the
    same attempts, r, n, the stored velocities, l, half_l and the clock, to 1e-10."""
    cells = colony(2000, 34, growth=1.5)
    cells[:, 13] = np.minimum(cells[:, 13], 4.0)      # no division in this iteration
    cells[:, 14] = cells[:, 13] / 2
    # a proposal that the error test rejects: BS3(2) is a third-order method, so its
    # errors pass up to larger steps than Heun-Euler's
    dt0, dt_max = {1: (1e-4, 2e-4), 2: (1e-3, 2e-3)}[mode]
    kw = dict(integration_mode=mode, max_stepsize=dt_max)
    if noise:
        kw.update(max_rxy_noise=50.0, max_rz_noise=20.0, max_nxy_noise=5.0, max_nz_noise=2.0)
    sim = abm_b200.Simulation(cap_cells=2100, jkr_table=JKR, controller=1, **kw)
    sim.upload_cells(cells)
    w = np.zeros(abm_b200.MLP_NPARAM, dtype=np.float32)
    w[-1] = 50.0                              # asks for 10x dt0; the proposal is clamped to dt_max
    sim.set_stepsize_weights(w)
    sim.set_clock(0.0, dt0, 0)
    sim.get_cell_neighbors()
    s = sim.iterate(1)
    assert s["iterations"] == 1 and s["rejected"] == 1
    o = orc.Oracle(dict(sim.pdict, controller=0), jkr=JKR)
    o.set_cells(cells)
    o.loop_init()
    o.set_clock(0.0, dt_max, 0)               # the reference rule's trial at the proposed dt
    o.iterate(1)
    so = o.stats()
    assert s["attempts"] == so["attempts"] and s["attempts"] >= 2
    t, dt, it = sim.clock()
    to, dto, ito = o.clock()
    assert it == ito == 1
    assert abs(dt - dto) <= 1e-12 * dto and abs(t - to) <= 1e-12 * to
    assert abs(s["last_max_error"] - so["last_max_error"]) <= 1e-9 * so["last_max_error"]
    got, ref = sim.download_cells(), o.cells()
    for c in range(1, 15):                    # r, n, stored velocities, l, half_l
        scale = np.abs(ref[:, c]).max()
        assert np.abs(got[:, c] - ref[:, c]).max() <= 1e-10 * max(scale, 1e-300), c
    assert np.array_equal(got[:, 15:], ref[:, 15:])
    sim.close()


@pytest.mark.parametrize("mode", [1, 2])
def test_pi_controller_matches_the_oracle(mode):
    """The PI controller (proposal dt 0.9 E_n^(-0.7/k) E_(n-1)^(0.4/k), a passing proposal
    accepted as is, the reference rule after a failing one) against the oracle's
    restatement over 30 iterations of a growing colony whose dt climbs from 1e-6 h to
    where the error test binds: the same attempts and rejections, the clock to 1e-6 and
    the cells to 1e-7.  Here dt follows E from step to step, and E is a cancellation:
    for the orientations the embedded error dt sum (b - b*) k is ~1e-6 of the step
    dt sum b k, so velocities that agree to ~1e-13 give E, and the next dt, to ~1e-7."""
    cells = colony(1500, 35, growth=1.5)
    cells[:, 13] = np.minimum(cells[:, 13], 4.0)
    cells[:, 14] = cells[:, 13] / 2
    sim = abm_b200.Simulation(cap_cells=1600, jkr_table=JKR, controller=abm_b200.CONTROLLER_PI,
                              integration_mode=mode, max_stepsize=1e-4, iter_update_neighbors=10)
    sim.upload_cells(cells)
    sim.set_clock(0.0, 1e-6, 0)
    sim.get_cell_neighbors()
    o = orc.Oracle(sim.pdict, jkr=JKR)
    o.set_cells(cells)
    o.loop_init()
    o.set_clock(0.0, 1e-6, 0)
    for _ in range(3):
        s = sim.iterate(10)
        o.iterate(10)
        so = o.stats()
        assert s["attempts"] == so["attempts"] and s["rejected"] == so["rejected"]
        t, dt, it = sim.clock()
        to, dto, ito = o.clock()
        assert it == ito and abs(t - to) <= 1e-6 * to and abs(dt - dto) <= 1e-6 * dto
        got, ref = sim.download_cells(), o.cells()
        for c in range(1, 15):
            scale = np.abs(ref[:, c]).max()
            assert np.abs(got[:, c] - ref[:, c]).max() <= 1e-7 * max(scale, 1e-300), c
    assert dt > 2e-6                          # the step grew from 1e-6 h to where the error test binds
    assert s["attempts"] < 2 * s["iterations"]   # passing proposals take one attempt
    sim.close()


def test_learned_controller_gain_over_pi_and_the_reference_controller():
    """What the trained network gains over the methods without it, at equal RK tolerance
    (1e-8) on growing, dividing colonies: RK evaluations per simulated hour, on three
    colonies of 2500 cells over 2000 steps.  The comparisons are the plain PI controller
    (the learned controller's baseline and fallback), the network with zero weights, and
    the reference rule (simulation.hpp:1688-1769).  The error test decides every step in
    all of them; rejected first attempts are counted in the evaluations and reported."""
    runs = [(stepsize.growing_colony(1500, 41), dict(max_stepsize=1e-4)),
            (stepsize.growing_colony(3000, 42), dict(max_stepsize=1e-4))]
    w, info = stepsize.train_protocol(runs, n_iters=1500, epochs=150)
    zero = np.zeros(abm_b200.MLP_NPARAM, np.float32)
    print("\nstep-size controllers on 2500-cell growing colonies, 2000 steps, tol 1e-8:")
    for seed in (43, 44, 45):
        cells = stepsize.growing_colony(2500, seed)
        res = {}
        for name, ctl, wt in (("reference", 0, None), ("pi", 2, None), ("zeroed", 1, zero), ("learned", 1, w)):
            rows, s = stepsize.logged_run(cells, 2000, controller=ctl, weights=wt)
            res[name] = s
            print("  seed %d %-9s evals/step %.3f  rejected %3d  t %.5f h  evals per h %.0f" % (
                seed, name, s["attempts"] / s["iterations"], s["rejected"], s["t"], s["attempts"] / s["t"]))
        eph = {k: s["attempts"] / s["t"] for k, s in res.items()}
        lrn, ref = res["learned"], res["reference"]
        # reference rule: trial + final every step, plus its retries; the proposing
        # controllers: one attempt per passing proposal, the reference rule after a failing one
        assert ref["attempts"] == 2 * ref["iterations"] + ref["retries"]
        for k in ("pi", "zeroed", "learned"):
            s = res[k]
            assert s["attempts"] == s["iterations"] + s["rejected"] + s["retries"]
        assert lrn["rejected"] <= 0.05 * lrn["iterations"]
        assert eph["learned"] <= 0.9 * eph["pi"], (seed, eph)
        assert eph["learned"] <= 0.9 * eph["zeroed"], (seed, eph)
        assert eph["learned"] <= 0.7 * eph["reference"], (seed, eph)
