"""CPU oracle of the learned block order's scorer and of its block features.

TEST INFRASTRUCTURE: only tests/ import this module; the product computes features in
ltl-learning-on-gpus_b200/csrc/order.cuh and runs the scorer with its own CUDA kernels
(csrc/mlp.cu, and the planner's warp scorer in csrc/ltl_kernels.cu).

The reference (MojtabaValizadeh/ltl-learning-on-gpus) has no learned component; what this
restates is the definition the CUDA kernels implement:

  * block features: order.cuh `block_features` (32 values from a block's operator, costs,
    operand sizes, and row statistics of its operand levels: how many stored rows hold at
    position 0 on every positive trace, and on no negative trace);
  * the scorer: a multilayer perceptron 32 -> 64 -> 64 -> 1 with ReLU, inputs, weights and
    activations rounded to BF16 (round to nearest even), products and sums in FP32;
  * the loss: mean over records of w * BCE-with-logits, w = pos_weight on label-1 records;
  * the gradient: backpropagation with the BF16 rounding points of mlp.cu (dz rounded for
    the W3 product, dh2 and dh1 rounded before their products).

`grad_exact` is the same network without any rounding, in float64, for finite-difference
checks of the backward formulas.
"""
from __future__ import annotations

import numpy as np

NF, H = 32, 64
W1, B1 = 0, H * NF
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H
PARAMS = B3 + 1


def bf16(x) -> np.ndarray:
    """Round float32 values to BF16 (round to nearest, ties to even); returned as float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)
    nan = np.isnan(a)
    if nan.any():
        out = np.where(nan, a, out)
    return out.reshape(a.shape)


def unpack(p):
    p = np.asarray(p, dtype=np.float32)
    return (p[W1:B1].reshape(H, NF), p[B1:W2], p[W2:B2].reshape(H, H), p[B2:W3], p[W3:B3], p[B3])


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases (float32)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, dtype=np.float32)
    p[W1:B1] = rng.normal(0.0, np.sqrt(2.0 / NF), H * NF)
    p[W2:B2] = rng.normal(0.0, np.sqrt(2.0 / H), H * H)
    p[W3:B3] = rng.normal(0.0, np.sqrt(1.0 / H), H)
    return p


def _forward(p, X):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    w1b, w2b, w3b = (bf16(w).astype(np.float64) for w in (w1, w2, w3))
    xb = bf16(np.asarray(X, dtype=np.float32)).astype(np.float64)
    a1 = xb @ w1b.T + b1
    h1 = bf16(np.maximum(a1, 0.0).astype(np.float32)).astype(np.float64)
    a2 = h1 @ w2b.T + b2
    h2 = bf16(np.maximum(a2, 0.0).astype(np.float32)).astype(np.float64)
    z = h2 @ w3b + float(b3)
    return xb, h1, h2, z, (w1b, w2b, w3b)


def forward(p, X) -> np.ndarray:
    """Logits of the BF16 scorer."""
    return _forward(p, X)[3]


def _bce(z, y, w):
    return w * (np.maximum(z, 0.0) - z * y + np.log1p(np.exp(-np.abs(z))))


def grad(p, X, Y, pos_weight: float = 1.0):
    """(gradient float64 [PARAMS], mean loss) with the BF16 rounding points of mlp.cu."""
    Y = np.asarray(Y, dtype=np.float64)
    xb, h1, h2, z, (w1b, w2b, w3b) = _forward(p, X)
    n = len(Y)
    w = np.where(Y > 0.5, pos_weight, 1.0)
    loss = float(_bce(z, Y, w).mean())
    dz = (w * (1.0 / (1.0 + np.exp(-z)) - Y) / n).astype(np.float32).astype(np.float64)
    dzb = bf16(dz.astype(np.float32)).astype(np.float64)
    dh2 = np.where(h2 > 0, bf16((dz[:, None] * w3b[None, :]).astype(np.float32)).astype(np.float64), 0.0)
    dh1 = np.where(h1 > 0, bf16((dh2 @ w2b).astype(np.float32)).astype(np.float64), 0.0)
    g = np.zeros(PARAMS, dtype=np.float64)
    g[W1:B1] = (dh1.T @ xb).ravel()
    g[B1:W2] = dh1.sum(0)
    g[W2:B2] = (dh2.T @ h1).ravel()
    g[B2:W3] = dh2.sum(0)
    g[W3:B3] = dzb @ h2
    g[B3] = dz.sum()
    return g, loss


def loss_exact(p, X, Y, pos_weight: float = 1.0) -> float:
    """Mean weighted BCE of the unrounded network (float64 throughout)."""
    p = np.asarray(p, dtype=np.float64)
    w1, b1 = p[W1:B1].reshape(H, NF), p[B1:W2]
    w2, b2 = p[W2:B2].reshape(H, H), p[B2:W3]
    w3, b3 = p[W3:B3], p[B3]
    X = np.asarray(X, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    h1 = np.maximum(X @ w1.T + b1, 0.0)
    h2 = np.maximum(h1 @ w2.T + b2, 0.0)
    z = h2 @ w3 + b3
    return float(_bce(z, Y, np.where(Y > 0.5, pos_weight, 1.0)).mean())


def grad_exact(p, X, Y, pos_weight: float = 1.0):
    """Gradient of loss_exact (float64, no rounding)."""
    p = np.asarray(p, dtype=np.float64)
    w1, b1 = p[W1:B1].reshape(H, NF), p[B1:W2]
    w2, b2 = p[W2:B2].reshape(H, H), p[B2:W3]
    w3, b3 = p[W3:B3], p[B3]
    X = np.asarray(X, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    n = len(Y)
    a1 = X @ w1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ w2.T + b2
    h2 = np.maximum(a2, 0.0)
    z = h2 @ w3 + b3
    w = np.where(Y > 0.5, pos_weight, 1.0)
    dz = w * (1.0 / (1.0 + np.exp(-z)) - Y) / n
    dh2 = (dz[:, None] * w3[None, :]) * (a2 > 0)
    dh1 = (dh2 @ w2) * (a1 > 0)
    g = np.zeros(PARAMS, dtype=np.float64)
    g[W1:B1] = (dh1.T @ X).ravel()
    g[B1:W2] = dh1.sum(0)
    g[W2:B2] = (dh2.T @ h1).ravel()
    g[B2:W3] = dh2.sum(0)
    g[W3:B3] = dz @ h2
    g[B3] = dz.sum()
    return g


# ---------------------------------------------------------------- block features (order.cuh)
def lg2lin(x: int) -> np.float32:
    if x <= 0:
        return np.float32(0.0)
    k = int(x).bit_length() - 1
    p = 1 << k
    return np.float32(np.float32(k) + np.float32(np.float32(x - p) / np.float32(p)))


def ratio(a: int, b: int) -> np.float32:
    return np.float32(np.float32(a) / np.float32(b)) if b > 0 else np.float32(0.0)


def block_features(op, cost, c1, lcost, rcost, position, nblocks, lrows, rrows, candidates, level_cands, lstat,
                   rstat, npos, nneg, nalpha) -> np.ndarray:
    """The 32 features of order.cuh, value by value in float32."""
    f = np.zeros(NF, dtype=np.float32)
    if 0 <= op < 7:
        f[op] = 1.0
    binary = op in (1, 2, 6)
    c = np.float32(cost)
    f[7] = c / np.float32(16.0)
    f[8] = np.float32(lcost) / c
    f[9] = np.float32(rcost) / c
    f[10] = lg2lin(lrows) / np.float32(24.0)
    f[11] = lg2lin(rrows) / np.float32(24.0)
    f[12] = lg2lin(candidates) / np.float32(32.0)
    f[13] = ratio(candidates, level_cands)
    f[14] = ratio(position, nblocks)
    f[15] = lg2lin(level_cands) / np.float32(32.0)
    for k in range(2):
        f[16 + k] = lg2lin(lstat[k] + 1) / np.float32(24.0)
        f[18 + k] = ratio(lstat[k], lrows)
        f[20 + k] = lg2lin(rstat[k] + 1) / np.float32(24.0)
        f[22 + k] = ratio(rstat[k], rrows) if binary else 0.0
    f[24] = ratio(npos, npos + nneg)
    f[25] = lg2lin(npos + nneg) / np.float32(16.0)
    f[26] = np.float32(nalpha) / np.float32(8.0)
    f[27] = 1.0 if binary else 0.0
    f[28] = 1.0 if binary and lcost == rcost else 0.0
    f[29] = 1.0 if lcost == c1 else 0.0
    f[30] = 1.0 if binary and rcost == c1 else 0.0
    f[31] = 1.0
    return f
