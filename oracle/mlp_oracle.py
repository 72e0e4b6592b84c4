"""CPU oracle of the entry / L-budget network of panns_b200 — TEST
INFRASTRUCTURE ONLY (imported by tests/ to check the GPU results, never by the product).

Restates, in float64 numpy, the network, loss and gradient that the GPU
kernels of parallel_anns_b200/csrc/learned.cu compute (the parameter layout
and loss of include/panns_learned.h), and the per-query decision of the
batched inference (decide_kernel in parallel_anns_b200/csrc/learned.cu). The weight
matrices are rounded to BF16 (round to nearest, ties to even) exactly as the
GPU rounds them; everything else is float64 here and float32 on the GPU, so
the two agree to float32 accumulation error. No reference counterpart exists
(the reference has no learned part); `numeric_grad` pins the analytic
gradient by central differences.
"""
from __future__ import annotations

import numpy as np

H = 256


def param_count(d: int, R: int) -> int:
    return d * H + H + H * H + H + H * (R + 1) + R + 1


def unpack(params: np.ndarray, d: int, R: int):
    p = np.asarray(params)
    o = 0
    out = []
    for shape in ((d, H), (H,), (H, H), (H,), (H, R + 1), (R + 1,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    assert o == p.size
    return out


def pack(parts) -> np.ndarray:
    return np.concatenate([np.asarray(x, dtype=np.float64).ravel() for x in parts])


def bf16_round(a: np.ndarray) -> np.ndarray:
    """float32 -> nearest BF16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def init_params(d: int, R: int, seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases (float32)."""
    rng = np.random.default_rng(seed)
    W1 = rng.normal(0, np.sqrt(2.0 / d), (d, H))
    W2 = rng.normal(0, np.sqrt(2.0 / H), (H, H))
    W3 = rng.normal(0, np.sqrt(1.0 / H), (H, R + 1))
    return pack([W1, np.zeros(H), W2, np.zeros(H), W3, np.zeros(R + 1)]).astype(np.float32)


def forward(params, X, d, R, bf16=True):
    W1, b1, W2, b2, W3, b3 = unpack(params, d, R)
    rnd = bf16_round if bf16 else (lambda w: np.asarray(w, dtype=np.float64))
    W1, W2, W3 = rnd(W1), rnd(W2), rnd(W3)
    b1, b2, b3 = (np.asarray(b, dtype=np.float64) for b in (b1, b2, b3))
    X = np.asarray(X, dtype=np.float64)
    H1 = np.maximum(X @ W1 + b1, 0.0)
    H2 = np.maximum(H1 @ W2 + b2, 0.0)
    Z = H2 @ W3 + b3
    return H1, H2, Z, (W1, W2, W3)


def label_hist(cells: np.ndarray, R: int) -> np.ndarray:
    B, T = cells.shape
    P = np.zeros((B, R))
    np.add.at(P, (np.repeat(np.arange(B), T), cells.ravel().astype(np.int64)), 1.0)
    return P / T


def loss_grad(params, X, cells, y, d, R, lam, bf16=True):
    """Batch-mean loss and its gradient (float64, parameter layout)."""
    B = X.shape[0]
    H1, H2, Z, (W1, W2, W3) = forward(params, X, d, R, bf16)
    P = label_hist(cells, R)
    lg = Z[:, :R]
    mx = lg.max(1, keepdims=True)
    lse = mx[:, 0] + np.log(np.exp(lg - mx).sum(1))
    e = Z[:, R] - np.asarray(y, dtype=np.float64)
    loss = np.mean(lse - (P * lg).sum(1) + 0.5 * lam * e * e)
    dZ = np.empty_like(Z)
    dZ[:, :R] = (np.exp(lg - lse[:, None]) - P) / B
    dZ[:, R] = lam * e / B
    dW3 = H2.T @ dZ
    db3 = dZ.sum(0)
    dH2 = (dZ @ W3.T) * (H2 > 0)
    dW2 = H1.T @ dH2
    db2 = dH2.sum(0)
    dH1 = (dH2 @ W2.T) * (H1 > 0)
    dW1 = np.asarray(X, dtype=np.float64).T @ dH1
    db1 = dH1.sum(0)
    return loss, pack([dW1, db1, dW2, db2, dW3, db3])


def numeric_grad(params, X, cells, y, d, R, lam, idx, h=1e-6):
    """Central differences of the float64 loss (weights not rounded) at idx."""
    p = np.asarray(params, dtype=np.float64).copy()
    g = np.empty(len(idx))
    for j, i in enumerate(idx):
        old = p[i]
        p[i] = old + h
        lp, _ = loss_grad(p, X, cells, y, d, R, lam, bf16=False)
        p[i] = old - h
        lm, _ = loss_grad(p, X, cells, y, d, R, lam, bf16=False)
        p[i] = old
        g[j] = (lp - lm) / (2 * h)
    return g


def decide(params, X, d, R, reps, *, E, L_init, L_min, use_L, L_scale, min_conf, K, L, L_exp=1.0):
    """The per-query decision of the batched inference: (fallback, L_q, entries, n_plain,
    confidence, regressor output, logits)."""
    _, _, Z, _ = forward(params, X, d, R, True)
    out = []
    for z in Z:
        lg = z[:R]
        conf = 1.0 / np.exp(lg - lg.max()).sum()
        fb = not conf >= min_conf
        Lq = L
        if not fb and use_L:
            v = np.float32(L_scale) * np.exp(np.float32(L_exp) * z[R])
            lo = max(K, min(L_min, L))
            if v < L:
                Lq = max(lo, int(np.ceil(max(v, 0.0))))
        ent = []
        if not fb and E:
            order = np.lexsort((np.arange(R), -lg))
            ent = [int(reps[c]) for c in order[:min(E, 64, Lq)]]
        n_plain = Lq - len(ent)
        if ent:
            n_plain = min(n_plain, L_init)
        out.append((fb, Lq, ent, n_plain, conf, float(z[R]), lg))
    return out
