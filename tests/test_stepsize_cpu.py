"""Step-size network on the CPU: the restated backward is the gradient of the
network (finite differences in FP64), BF16 rounding is round-to-nearest-even,
and the training targets follow the error model of the controller."""
import numpy as np

import mlp_ref
from abm_b200 import stepsize


def rand_problem(n, seed):
    rng = np.random.default_rng(seed)
    w = stepsize.init_weights(seed, out_bias=0.1)
    w[mlp_ref.OFF_B1:mlp_ref.OFF_W2] = rng.normal(0, 0.1, 64)
    w[mlp_ref.OFF_B2:mlp_ref.OFF_W3] = rng.normal(0, 0.1, 64)
    X = rng.normal(0, 1, (n, 32)).astype(np.float32)
    T = rng.normal(0, 1, n).astype(np.float32)
    return w, X, T


def test_bf16_rounding_ties_to_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -9, -2.5, 3.0e-3, 65504.0],
                 dtype=np.float32)
    got = mlp_ref.bf16(x)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties go to the even mantissa (1.0)
    expect = np.array([1.0, 1.0, 1.0 + 2 * 2.0 ** -7, 1.0, -2.5, np.float32(3.0e-3), 65536.0], dtype=np.float32)
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == expect[2] and got[3] == 1.0 and got[4] == -2.5
    assert abs(got[5] - 3.0e-3) / 3.0e-3 < 2.0 ** -8
    assert got[6] == 65536.0
    assert np.all(mlp_ref.bf16(got) == got)                 # idempotent


def test_fp64_gradient_matches_finite_differences():
    w, X, T = rand_problem(37, 1)
    g, _ = mlp_ref.grad_fp64(w, X, T)
    rng = np.random.default_rng(2)
    idx = np.concatenate([rng.choice(np.arange(mlp_ref.OFF_W1, mlp_ref.OFF_B1), 12),
                          rng.choice(np.arange(mlp_ref.OFF_B1, mlp_ref.OFF_W2), 6),
                          rng.choice(np.arange(mlp_ref.OFF_W2, mlp_ref.OFF_B2), 12),
                          rng.choice(np.arange(mlp_ref.OFF_B2, mlp_ref.OFF_W3), 6),
                          rng.choice(np.arange(mlp_ref.OFF_W3, mlp_ref.OFF_B3), 6), [mlp_ref.OFF_B3]])
    w64 = w.astype(np.float64)
    for k in idx:
        h = 1e-6 * max(1.0, abs(w64[k]))
        wp, wm = w64.copy(), w64.copy()
        wp[k] += h
        wm[k] -= h
        fd = (mlp_ref.loss_fp64(wp, X, T) - mlp_ref.loss_fp64(wm, X, T)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])) + 1e-9, (k, fd, g[k])


def test_bf16_gradient_close_to_exact():
    w, X, T = rand_problem(64, 3)
    g, loss = mlp_ref.grad(w, X, T)
    g64, loss64 = mlp_ref.grad_fp64(w, X, T)
    assert abs(loss - loss64) <= 2e-2 * loss64
    assert np.linalg.norm(g - g64) <= 3e-2 * np.linalg.norm(g64)


def test_training_targets_follow_the_error_model():
    rows = np.zeros((4, 40), dtype=np.float32)
    rows[:, 36] = [0.0, 0.0, 0.0, 0.5]                         # error-model baseline b
    # HE21: dt_max = dt_first E^(-1/2); E = 0.25 -> ln(dt_max/dt_first) = ln 2
    rows[0, 32], rows[0, 33] = np.log(2.0), 0.0
    rows[1, 32], rows[1, 33] = np.log(2.0), np.log(0.5)      # the first attempt ran at half dt_prev
    rows[2, 32], rows[2, 33] = 34.5, 0.0                       # E floored at min_error: clamp at 10
    rows[3, 32], rows[3, 33] = -5.0, 0.0                       # E huge: clamp at 0.2
    X, T = stepsize.training_pairs(rows, safety=0.9)
    assert X.shape == (4, 32)
    np.testing.assert_allclose(T, [np.log(1.8), np.log(0.9), np.log(10.0), np.log(0.2) - 0.5], rtol=1e-6)
