"""Autotuner of the batched search: for one shape (index, batch of tuning
queries with their true neighbours, K, recall target) it picks the storage,
M (candidates expanded per step), the warps per block, the queue length L
(which also sets each warp's shared-memory queue capacity) and, when a
learned model is given, whether and how to use it, by measuring.

Procedure, per candidate (storage, M, learned option): the smallest L of a
grid whose recall on the tuning queries meets the target (binary search; the
recall of a search grows with L), then the block shape that runs it fastest:
warps per block and resident blocks per SM (which sets how much of each SM's
L1 / shared array is left to L1) with one warp per query, or 2 / 4 warps per
query (one query per block, for small batches); the fastest candidate wins. Times are the search kernel's CUDA-event
time, best of ``reps``. Evaluate the result on other queries than the tuning
ones. Choices are cached per shape in a JSON file when ``cache`` is given.
"""
from __future__ import annotations

import json
import os
from dataclasses import asdict, dataclass, field

import numpy as np

from . import native as N

L_GRID = (100, 120, 140, 160, 180, 200, 224, 256, 288, 320, 352, 384, 416, 448, 512, 576, 640, 720, 800,
          896, 1024, 1152, 1280, 1440, 1600, 1792, 2048, 2304, 2560, 3072, 4096, 4608, 5120, 6144, 8192)


@dataclass
class Choice:
    storage: int
    M: int
    L: int
    warps_per_block: int
    learned: dict | None = None      # options of learned.attach, or None for the plain search
    blocks_per_sm: int = 0           # resident blocks per SM (0 = as many as fit)
    warps_per_query: int = 1         # 1: one warp per query; 2 / 4: one query per block of that many warps
    recall: float = 0.0
    kernel_ms: float = 0.0
    qps: float = 0.0
    table: list = field(default_factory=list)

    def search_kwargs(self):
        from . import native as _N
        return dict(L=self.L, M=self.M, mode=_N.MODE_NSG_SEQ if self.M == 1 else _N.MODE_TOP_M,
                    storage=self.storage, warps_per_block=self.warps_per_block,
                    blocks_per_sm=self.blocks_per_sm, warps_per_query=self.warps_per_query,
                    flags=_N.FLAG_LEARNED if self.learned is not None else 0)


def _time(index, queries, K, kw, reps):
    best, ids = 1e30, None
    for _ in range(reps):
        ids, st = index.search(queries, K=K, **kw)
        best = min(best, st["kernel_ms"])
    return ids, best


def tune(index, queries, gt, *, K=100, target=0.95, storages=(N.STORE_FP32,), Ms=(1, 2, 4, 8, 16),
         wpbs=(2, 4), bpss=(0, 5, 4), wpqs=(1,), learned_model=None, learned_opts=(), include_plain=True,
         L_grid=L_GRID, reps=2, cache=None, log=None) -> Choice:
    from . import learned as LE
    from .searching import recall
    key = None
    if cache:
        key = json.dumps({"n": index.n, "d": index.d, "nq": int(queries.shape[0]), "K": K, "target": target,
                          "storages": list(storages), "Ms": list(Ms), "wpbs": list(wpbs), "bpss": list(bpss), "wpqs": list(wpqs),
                          "learned": [dict(o) for o in learned_opts] if learned_model is not None else [],
                          "plain": include_plain, "grid": list(L_grid)}, sort_keys=True)
        if os.path.exists(cache):
            with open(cache) as f:
                saved = json.load(f)
            if key in saved:
                return Choice(**saved[key])
    options = ([None] if include_plain else []) + (list(learned_opts) if learned_model is not None else [])
    table = []
    best = None
    for store in storages:
        for opt in options:
            if opt is not None:
                LE.attach(index, learned_model, **opt)
            for M in Ms:
                flags = N.FLAG_LEARNED if opt is not None else 0
                mode = N.MODE_NSG_SEQ if M == 1 else N.MODE_TOP_M
                kw = dict(M=M, mode=mode, storage=store, flags=flags, warps_per_block=0)
                rec_at = {}

                def rec(L):
                    if L not in rec_at:
                        ids, _ = index.search(queries, K=K, L=L, **kw)
                        rec_at[L] = recall(ids, gt, 100, 100)
                    return rec_at[L]

                lo, hi = 0, len(L_grid) - 1
                if rec(L_grid[hi]) < target:
                    table.append({"storage": store, "M": M, "learned": opt, "L": None, "recall": rec(L_grid[hi])})
                    continue
                while lo < hi:
                    mid = (lo + hi) // 2
                    if rec(L_grid[mid]) >= target:
                        hi = mid
                    else:
                        lo = mid + 1
                L = L_grid[lo]
                shapes = [(w, bps, 1) for w in wpbs for bps in bpss]
                shapes += [(wq, 0, wq) for wq in wpqs if wq > 1]  # several warps per query
                for w, bps, wq in shapes:
                    # blocks_per_sm counts blocks of w warps: keep the warps per SM comparable
                    b = bps * 4 // w if bps else 0
                    kw2 = dict(kw, warps_per_block=w, blocks_per_sm=b, warps_per_query=wq)
                    try:
                        _, ms = _time(index, queries, K, dict(kw2, L=L), reps)
                    except N.PannsError as e:  # a block shape that does not fit this L
                        if e.code != -1:
                            raise
                        continue
                    row = {"storage": store, "M": M, "learned": opt, "L": L, "warps_per_block": w,
                           "blocks_per_sm": b, "warps_per_query": wq, "recall": rec(L), "kernel_ms": ms}
                    table.append(row)
                    if best is None or ms < best.kernel_ms:
                        best = Choice(store, M, L, w, opt, b, wq, rec(L), ms, queries.shape[0] / (ms / 1e3))
                if log:
                    log(f"autotune storage={store} M={M} learned={opt}: L={L} recall={rec(L):.4f} "
                        f"ms={min(r['kernel_ms'] for r in table if r.get('L') == L and r['M'] == M and r['storage'] == store and r['learned'] == opt):.3f}")
    if best is None:
        raise RuntimeError("autotune: no configuration reaches the recall target")
    best.table = table
    if cache:
        saved = {}
        if os.path.exists(cache):
            with open(cache) as f:
                saved = json.load(f)
        saved[key] = asdict(best)
        os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
        with open(cache, "w") as f:
            json.dump(saved, f)
    if best.learned is not None:
        LE.attach(index, learned_model, **best.learned)
    return best
