"""CPU restatement of the step-size network (test infrastructure: the GPU forward,
backward and training kernels are compared against it; nothing in the product imports it).

The network is 32 -> 64 -> 64 -> 1 with ReLU, flat FP32 parameters
W1[64][32], b1[64], W2[64][64], b2[64], w3[64], b3.  The GPU kernels round the
operands of every tensor-core product to BF16 (round to nearest even) and
accumulate in FP32; this restatement rounds the same operands at the same points
and accumulates in FP64, so the two agree to FP32 accumulation error.

The reference has no counterpart (its controller is the rule of
simulation.hpp:1688-1769); the network is specified by the task, not by the
reference, so there is nothing to pin beyond the mathematics: `grad_fp64` is the
exact gradient of the unrounded network, checked by finite differences.
"""
import numpy as np

NIN, NH = 32, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + NH * NIN
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NH
NPARAM = OFF_B3 + 1


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(w, dtype=np.float32):
    w = np.asarray(w, dtype=dtype)
    return (w[OFF_W1:OFF_B1].reshape(NH, NIN), w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(NH, NH),
            w[OFF_B2:OFF_W3], w[OFF_W3:OFF_B3], w[OFF_B3])


def forward(w, X):
    """Outputs and hidden activations as the GPU computes them (BF16 operands)."""
    W1, b1, W2, b2, w3, b3 = unpack(w)
    X = np.asarray(X, dtype=np.float32)
    a1 = bf16(X).astype(np.float64) @ bf16(W1).astype(np.float64).T
    H1 = np.maximum((a1.astype(np.float32) + b1).astype(np.float32), 0)
    a2 = bf16(H1).astype(np.float64) @ bf16(W2).astype(np.float64).T
    H2 = np.maximum((a2.astype(np.float32) + b2).astype(np.float32), 0)
    a3 = bf16(H2).astype(np.float64) @ bf16(w3).astype(np.float64)
    y = (a3.astype(np.float32) + b3).astype(np.float32)
    return y, H1, H2


def grad(w, X, T):
    """Gradient of L = 0.5/n sum (y - t)^2 with the rounding points of the GPU
    backward: BF16 operands in every product with a weight matrix or an
    activation matrix, FP32 elsewhere; returns (grad, loss)."""
    W1, b1, W2, b2, w3, b3 = unpack(w)
    X = np.asarray(X, dtype=np.float32)
    T = np.asarray(T, dtype=np.float32)
    n = X.shape[0]
    y, H1, H2 = forward(w, X)
    loss = float(0.5 * np.sum((y.astype(np.float64) - T) ** 2) / n)
    dY = ((y - T) / np.float32(n)).astype(np.float32)
    g = np.zeros(NPARAM, dtype=np.float64)
    g[OFF_W3:OFF_B3] = dY.astype(np.float64) @ H2.astype(np.float64)
    g[OFF_B3] = dY.astype(np.float64).sum()
    dH2 = np.where(H2 > 0, dY[:, None] * bf16(w3)[None, :], 0).astype(np.float32)
    g[OFF_W2:OFF_B2] = (bf16(dH2).astype(np.float64).T @ bf16(H1).astype(np.float64)).ravel()
    g[OFF_B2:OFF_W3] = dH2.astype(np.float64).sum(axis=0)
    dH1 = (bf16(dH2).astype(np.float64) @ bf16(W2).astype(np.float64)).astype(np.float32)
    dH1 = np.where(H1 > 0, dH1, 0).astype(np.float32)
    g[OFF_W1:OFF_B1] = (bf16(dH1).astype(np.float64).T @ bf16(X).astype(np.float64)).ravel()
    g[OFF_B1:OFF_W2] = dH1.astype(np.float64).sum(axis=0)
    return g, loss


def forward_fp64(w, X):
    W1, b1, W2, b2, w3, b3 = unpack(w, np.float64)
    H1 = np.maximum(np.asarray(X, np.float64) @ W1.T + b1, 0)
    H2 = np.maximum(H1 @ W2.T + b2, 0)
    return H2 @ w3 + b3, H1, H2


def grad_fp64(w, X, T):
    """Exact gradient of the unrounded network in FP64 (same formulas as `grad`)."""
    W1, b1, W2, b2, w3, b3 = unpack(w, np.float64)
    X = np.asarray(X, np.float64)
    n = X.shape[0]
    y, H1, H2 = forward_fp64(w, X)
    dY = (y - np.asarray(T, np.float64)) / n
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = dY @ H2
    g[OFF_B3] = dY.sum()
    dH2 = np.where(H2 > 0, dY[:, None] * w3[None, :], 0)
    g[OFF_W2:OFF_B2] = (dH2.T @ H1).ravel()
    g[OFF_B2:OFF_W3] = dH2.sum(axis=0)
    dH1 = np.where(H1 > 0, dH2 @ W2, 0)
    g[OFF_W1:OFF_B1] = (dH1.T @ X).ravel()
    g[OFF_B1:OFF_W2] = dH1.sum(axis=0)
    return g, float(0.5 * np.sum((y - np.asarray(T, np.float64)) ** 2) / n)


def loss_fp64(w, X, T):
    y, _, _ = forward_fp64(w, X)
    return 0.5 * np.sum((y - np.asarray(T, np.float64)) ** 2) / X.shape[0]
