"""CPU restatement (numpy, FP64) of the block-size selector network, used only
as the checker of the GPU selector kernels (test infrastructure: nothing in
the product path imports it).

The selector has no reference code: the reference picks blocks from fixed
policies (``double_blocked_potrf.cpp:17-20, 232-233``; the tuned
``docs/numerical_validation.md:64-65`` values) and its benchmark cases sweep
(nb, b) by hand (``src/potrf/benchmark/potrf_double_blocked_cases.cpp``).
The network restated here is this repository's own design:

    h1 = relu(x W1 + b1)          x: F features, W1: F x H
    h2 = relu(h1 W2 + b2)         W2: H x H
    z  = h2 W3 + b3               W3: H x K candidate scores
    p  = softmax(z over the valid candidates of the sample)
    loss = mean_s  sum_k -q_sk log p_sk

q is the soft target built from measured times (``soft_targets``).  The flat
parameter layout is [W1 (row-major F x H), b1, W2 (H x H), b2, W3 (H x K), b3],
identical to the device layout.  Adam (beta1 0.9, beta2 0.999, eps 1e-8) with
L2 weight decay folded into the gradient.
"""
from __future__ import annotations

import numpy as np

from . import uniform_pm1

HIDDEN = 64


def n_params(F: int, K: int, H: int = HIDDEN) -> int:
    return F * H + H + H * H + H + H * K + K


def unpack(theta: np.ndarray, F: int, K: int, H: int = HIDDEN):
    o = 0
    out = []
    for shape in [(F, H), (H,), (H, H), (H,), (H, K), (K,)]:
        size = int(np.prod(shape))
        out.append(theta[o:o + size].reshape(shape))
        o += size
    return out


def init_params(F: int, K: int, seed: int, H: int = HIDDEN) -> np.ndarray:
    """Glorot-uniform weights from the counter-based U[-1,1) stream, zero
    biases (FP32, bit-identical to the device initialiser)."""
    theta = uniform_pm1(n_params(F, K, H), seed).astype(np.float32)
    W1, b1, W2, b2, W3, b3 = unpack(theta, F, K, H)
    for W, fi, fo in [(W1, F, H), (W2, H, H), (W3, H, K)]:
        s = np.sqrt(np.float32(6.0) / np.float32(fi + fo)).astype(np.float32)
        W *= s
    for b in (b1, b2, b3):
        b[:] = 0
    return theta


def forward(theta, X, mask, F, K, H=HIDDEN):
    W1, b1, W2, b2, W3, b3 = [np.asarray(a, dtype=np.float64) for a in unpack(theta, F, K, H)]
    X = np.asarray(X, dtype=np.float64)
    a1 = X @ W1 + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2 + b2
    h2 = np.maximum(a2, 0.0)
    z = h2 @ W3 + b3
    valid = np.asarray(mask) > 0
    zm = np.where(valid, z, -np.inf)
    zmax = zm.max(axis=1, keepdims=True)
    e = np.where(valid, np.exp(zm - zmax), 0.0)
    p = e / e.sum(axis=1, keepdims=True)
    return p, (X, h1, h2, valid)


def loss_and_grad(theta, X, Q, mask, F, K, H=HIDDEN):
    """Mean masked cross-entropy and its gradient (flat, FP64)."""
    W1, b1, W2, b2, W3, b3 = [np.asarray(a, dtype=np.float64) for a in unpack(theta, F, K, H)]
    p, (Xd, h1, h2, valid) = forward(theta, X, mask, F, K, H)
    N = Xd.shape[0]
    Qd = np.where(valid, np.asarray(Q, dtype=np.float64), 0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        logp = np.where(valid, np.log(np.where(valid, p, 1.0)), 0.0)
    loss = float(-(Qd * logp).sum() / N)
    dz = np.where(valid, p - Qd, 0.0) / N
    gW3 = h2.T @ dz
    gb3 = dz.sum(0)
    dh2 = (dz @ W3.T) * (h2 > 0)
    gW2 = h1.T @ dh2
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (h1 > 0)
    gW1 = Xd.T @ dh1
    gb1 = dh1.sum(0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return loss, g


def adam_train(theta, X, Q, mask, F, K, epochs, lr, wd=1e-4, H=HIDDEN):
    """Full-batch Adam; returns (theta, losses).  FP64 restatement of the
    device training loop."""
    th = np.asarray(theta, dtype=np.float64).copy()
    m = np.zeros_like(th)
    v = np.zeros_like(th)
    losses = []
    for t in range(1, epochs + 1):
        loss, g = loss_and_grad(th, X, Q, mask, F, K, H)
        losses.append(loss)
        g = g + wd * th
        m = 0.9 * m + 0.1 * g
        v = 0.999 * v + 0.001 * g * g
        mh = m / (1 - 0.9 ** t)
        vh = v / (1 - 0.999 ** t)
        th -= lr * mh / (np.sqrt(vh) + 1e-8)
    return th, losses


def soft_targets(times, mask, tau=0.02):
    """q_k proportional to exp(-(t_k / t_best - 1) / tau) over valid
    candidates: the fastest candidate dominates, near-ties share mass."""
    t = np.where(np.asarray(mask) > 0, np.asarray(times, dtype=np.float64), np.inf)
    best = t.min(axis=1, keepdims=True)
    s = np.where(np.isfinite(t), np.exp(-(t / best - 1.0) / tau), 0.0)
    return s / s.sum(axis=1, keepdims=True)


def numeric_grad(theta, X, Q, mask, F, K, idx, h=1e-6, H=HIDDEN):
    """Central differences of the loss for the parameters in idx (FP64)."""
    th = np.asarray(theta, dtype=np.float64)
    out = []
    for i in idx:
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        lp, _ = loss_and_grad(tp, X, Q, mask, F, K, H)
        lm, _ = loss_and_grad(tm, X, Q, mask, F, K, H)
        out.append((lp - lm) / (2 * h))
    return np.array(out)
