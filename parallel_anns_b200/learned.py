"""Learned entry vertices and per-query L budget for the batched search.

Pipeline (every numeric step runs on the GPU through the C ABI of
include/panns_learned.h):

1. ``kmeans``: R representatives of the base (Lloyd k-means; each cell's
   vertex nearest its centroid).
2. ``traces``: the plain method labels held-out training queries. Its
   top-K result at a large queue length stands for the query's neighbours;
   the cells of the nearest T of them are the entry target (a histogram over
   the R representatives), and the smallest L of a grid whose plain search
   reaches the recall target against those neighbours is the L-budget target
   (y = ln L).
3. ``train``: Adam on the network x -> relu 256 -> relu 256 -> (R logits,
   1 L output), BF16 weights, float32 accumulation, by the library's own
   forward / backward kernels.
4. ``attach``: hands the network and representatives to an ``Index``;
   searches with ``flags=FLAG_LEARNED`` then run it batched before the search
   kernel and start each query from its decision,
   and queries whose top softmax probability is below ``min_conf`` run the
   plain search (PANNS init list, the call's L).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

from . import native as N

H = 256


def param_count(d: int, R: int) -> int:
    return int(N.load().panns_mlp_param_count(d, R))


def init_params(d: int, R: int, seed: int = 0, y_mean: float = 0.0) -> np.ndarray:
    """He-normal weights, zero biases; the L output's bias starts at y_mean."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0, np.sqrt(2.0 / d), (d, H)), np.zeros(H),
             rng.normal(0, np.sqrt(2.0 / H), (H, H)), np.zeros(H),
             rng.normal(0, np.sqrt(1.0 / H), (H, R + 1)), np.zeros(R + 1)]
    parts[5][R] = y_mean
    p = np.concatenate([np.asarray(x, dtype=np.float64).ravel() for x in parts]).astype(np.float32)
    assert p.size == param_count(d, R)
    return p


@dataclass
class LearnedModel:
    d: int
    R: int
    params: np.ndarray              # float32, layout of include/panns_learned.h
    reps: np.ndarray                # R original ids
    info: dict = field(default_factory=dict)

    def save(self, path: str):
        np.savez(path, d=self.d, R=self.R, params=self.params, reps=self.reps)

    @staticmethod
    def load(path: str) -> "LearnedModel":
        z = np.load(path)
        return LearnedModel(int(z["d"]), int(z["R"]), z["params"].astype(np.float32),
                            z["reps"].astype(np.uint32))


def kmeans(index, R: int = 1024, iters: int = 15, seed: int = 1):
    """Representatives (R original ids) and the cell of every base vertex."""
    reps = np.empty(R, dtype=np.uint32)
    assign = np.empty(index.n, dtype=np.uint32)
    N.check(N.load().panns_kmeans(index._h, R, iters, seed, N.ptr(reps), N.ptr(assign), None))
    return reps, assign


DEFAULT_L_GRID = (100, 120, 150, 180, 220, 270, 330, 400, 500, 650, 800)


def traces(index, queries, assign, *, K=100, M=8, L_ref=1000, T=10, L_grid=DEFAULT_L_GRID,
           recall_target=0.95, chunk=50_000):
    """Training labels from the plain method: (cells [n x T] uint16,
    y [n] float32 = ln of the smallest grid L reaching the recall target,
    Lmin [n])."""
    n = queries.shape[0]
    cells = np.empty((n, T), dtype=np.uint16)
    Lmin = np.full(n, int(L_grid[-1] * 1.25), dtype=np.int64)
    for s in range(0, n, chunk):
        q = queries[s:s + chunk]
        ref, _ = index.search(q, K=K, L=L_ref, mode=N.MODE_TOP_M, M=M)
        cells[s:s + chunk] = assign[ref[:, :T]].astype(np.uint16)
        done = np.zeros(q.shape[0], dtype=bool)
        for L in L_grid:
            ids, _ = index.search(q, K=K, L=L, mode=N.MODE_TOP_M, M=M)
            hit = per_query_recall(ids, ref, K) >= recall_target
            new = hit & ~done
            Lmin[s:s + chunk][new] = L
            done |= hit
    y = np.log(Lmin).astype(np.float32)
    return cells, y, Lmin


def per_query_recall(ids: np.ndarray, ref: np.ndarray, K: int) -> np.ndarray:
    """|ids[i] ∩ ref[i, :K]| / K per row."""
    a = np.sort(ids[:, :K].astype(np.int64), 1)
    b = np.sort(ref[:, :K].astype(np.int64), 1)
    off = (np.arange(a.shape[0], dtype=np.int64) * (1 << 32))[:, None]
    inter = np.isin(a + off, b + off, assume_unique=True).sum(1)
    return inter / float(K)


def train(X, cells, y, R, *, epochs=8, batch=1024, lr=2e-3, lam=1.0, weight_decay=0.0, seed=0,
          device=0, params=None):
    """Train on the GPU; returns (params, per-epoch mean loss)."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    cells = np.ascontiguousarray(cells, dtype=np.uint16)
    y = np.ascontiguousarray(y, dtype=np.float32)
    n, d = X.shape
    if params is None:
        params = init_params(d, R, seed, float(y.mean()))
    params = np.ascontiguousarray(params, dtype=np.float32).copy()
    tp = N.MlpTrainParams(d, R, cells.shape[1], batch, epochs, seed, lr, 0.9, 0.999, 1e-8, weight_decay, lam)
    losses = np.zeros(epochs, dtype=np.float64)
    N.check(N.load().panns_mlp_train(device, ctypes.byref(tp), N.ptr(X), N.ptr(cells), N.ptr(y), n,
                                     N.ptr(params), N.ptr(losses)))
    return params, losses


def loss_grad(params, X, cells, y, R, lam=1.0, device=0):
    """Loss and gradient of one batch by the GPU kernels."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    cells = np.ascontiguousarray(cells, dtype=np.uint16)
    y = np.ascontiguousarray(y, dtype=np.float32)
    params = np.ascontiguousarray(params, dtype=np.float32)
    B, d = X.shape
    grad = np.empty(params.size, dtype=np.float32)
    loss = ctypes.c_double()
    N.check(N.load().panns_mlp_loss_grad(device, d, R, cells.shape[1], N.ptr(params), N.ptr(X), N.ptr(cells),
                                         N.ptr(y), B, lam, N.ptr(grad), ctypes.byref(loss)))
    return loss.value, grad


def forward(params, X, R, device=0):
    X = np.ascontiguousarray(X, dtype=np.float32)
    params = np.ascontiguousarray(params, dtype=np.float32)
    n, d = X.shape
    Z = np.empty((n, R + 1), dtype=np.float32)
    N.check(N.load().panns_mlp_forward(device, d, R, N.ptr(params), N.ptr(X), n, N.ptr(Z)))
    return Z


def attach(index, model: LearnedModel, *, E=16, L_init=1 << 30, L_min=0, use_L=True, L_scale=1.0,
           L_exp=1.0, min_conf=0.0):
    lp = N.LearnedParams(E, min(L_init, 0xFFFFFFFF), L_min, 1 if use_L else 0, L_scale, L_exp, min_conf)
    params = np.ascontiguousarray(model.params, dtype=np.float32)
    reps = np.ascontiguousarray(model.reps, dtype=np.uint32)
    N.check(N.load().panns_set_learned(index._h, N.ptr(params), model.R, N.ptr(reps), ctypes.byref(lp)))


REC_WORDS = 66


def record(index, nq: int):
    """Per query of the last learned search: (L used, fallback flag, entries)."""
    out = np.empty((nq, REC_WORDS), dtype=np.uint32)
    N.check(N.load().panns_learned_record(index._h, nq, N.ptr(out)))
    Lq = (out[:, 0] & 0x7FFFFFFF).astype(np.int64)
    fb = (out[:, 0] >> 31).astype(bool)
    entries = [out[i, 2:2 + out[i, 1]].copy() for i in range(nq)]
    return Lq, fb, entries


def build_model(index, train_queries, *, R=1024, K=100, M=8, L_ref=1000, T=10, epochs=8, batch=1024,
                lr=2e-3, lam=1.0, seed=0, kmeans_iters=15, cache=None, log=None):
    """k-means + traces + training, cached in the .npz ``cache`` if given."""
    if cache and os.path.exists(cache):
        return LearnedModel.load(cache)
    reps, assign = kmeans(index, R, kmeans_iters, seed + 1)
    cells, y, Lmin = traces(index, train_queries, assign, K=K, M=M, L_ref=L_ref, T=T)
    params, losses = train(train_queries, cells, y, R, epochs=epochs, batch=batch, lr=lr, lam=lam, seed=seed)
    m = LearnedModel(train_queries.shape[1], R, params, reps,
                     {"losses": losses.tolist(), "Lmin_hist": np.unique(Lmin, return_counts=True)})
    if log:
        log(f"learned model: R={R}, {train_queries.shape[0]} training queries, losses {np.round(losses, 4)}")
    if cache:
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        m.save(cache)
    return m
