"""Readers and writers for the on-disk formats of PANNS's search path.

All formats are little-endian and bit-compatible with the reference:

* fvecs: per row ``u32 d`` then ``d x f32``
  (reader: ``include/utils.h:95-138`` ``DiskIO::load_data``).
* .nsg: ``u32 width, u32 entry``, then per vertex ``u32 degree`` followed by
  ``degree x u32`` neighbour ids (writer: ``include/efanna2e/index_nsg.cpp:20-32``
  ``IndexNSG::Save``; readers ``core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp:57-133``
  and ``core/Searching.202102031939.PSS_v5.large_graph.dist_thresh.profiling.cpp:138-258``).
* true-NN: ``u32 nq, u32 K``, then ``nq x K x (u32 id, f32 dist)``
  (writer: ``tools/save_true_nearest_neighbors.cpp:37-64``; reader:
  ``core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp:141-189``).
* results: per query ``u32 K`` then ``K x u32`` (``include/utils.h:146-160``
  ``DiskIO::save_result``).
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np


def write_fvecs(path: str, x: np.ndarray) -> None:
    x = np.ascontiguousarray(x, dtype=np.float32)
    n, d = x.shape
    rec = np.empty((n, d + 1), dtype=np.float32)
    rec[:, 0] = np.array([d], dtype=np.uint32).view(np.float32)[0]
    rec[:, 1:] = x
    rec.tofile(path)


def read_fvecs(path: str) -> np.ndarray:
    raw = np.fromfile(path, dtype=np.uint32)
    if raw.size == 0:
        return np.zeros((0, 0), dtype=np.float32)
    d = int(raw[0])
    if raw.size % (d + 1):
        raise ValueError(f"{path}: size {raw.size * 4} B is not a whole number of {d}-d rows")
    rec = raw.reshape(-1, d + 1)
    if not np.all(rec[:, 0] == d):
        raise ValueError(f"{path}: rows disagree on the dimension")
    return rec[:, 1:].view(np.float32).copy()


@dataclass
class NSGGraph:
    """An NSG graph in CSR form: ``offsets[v]..offsets[v+1]`` index ``nbrs``."""

    width: int
    entry: int
    offsets: np.ndarray  # int64 [N+1]
    nbrs: np.ndarray  # uint32 [E]

    @property
    def n(self) -> int:
        return int(self.offsets.shape[0] - 1)

    def degree(self) -> np.ndarray:
        return np.diff(self.offsets).astype(np.uint32)

    def neighbors(self, v: int) -> np.ndarray:
        return self.nbrs[self.offsets[v]:self.offsets[v + 1]]

    @staticmethod
    def from_lists(width: int, entry: int, lists) -> "NSGGraph":
        deg = np.array([len(l) for l in lists], dtype=np.int64)
        off = np.zeros(len(lists) + 1, dtype=np.int64)
        np.cumsum(deg, out=off[1:])
        nb = np.concatenate([np.asarray(l, dtype=np.uint32) for l in lists]) if len(lists) else \
            np.zeros(0, dtype=np.uint32)
        return NSGGraph(int(width), int(entry), off, nb.astype(np.uint32))


def write_nsg(path: str, g: NSGGraph) -> None:
    deg = g.degree()
    n = g.n
    out = np.empty(2 + n + g.nbrs.shape[0], dtype=np.uint32)
    out[0] = g.width
    out[1] = g.entry
    # Row v starts at 2 + offsets[v] + v (one degree word per earlier row).
    starts = 2 + g.offsets[:-1] + np.arange(n, dtype=np.int64)
    out[starts] = deg
    mask = np.ones(out.shape[0], dtype=bool)
    mask[:2] = False
    mask[starts] = False
    out[mask] = g.nbrs
    out.tofile(path)


def read_nsg(path: str) -> NSGGraph:
    raw = np.fromfile(path, dtype=np.uint32)
    if raw.size < 2:
        raise ValueError(f"{path}: truncated header")
    width, entry = int(raw[0]), int(raw[1])
    degs = []
    pos = 2
    total = raw.size
    # Walk the rows; vectorised walking is not possible without the degrees.
    while pos < total:
        d = int(raw[pos])
        if pos + 1 + d > total:
            raise ValueError(f"{path}: truncated row at word {pos}")
        degs.append(d)
        pos += 1 + d
    deg = np.array(degs, dtype=np.int64)
    off = np.zeros(deg.shape[0] + 1, dtype=np.int64)
    np.cumsum(deg, out=off[1:])
    starts = 2 + off[:-1] + np.arange(deg.shape[0], dtype=np.int64)
    mask = np.ones(total, dtype=bool)
    mask[:2] = False
    mask[starts] = False
    return NSGGraph(width, entry, off, raw[mask].copy())


def write_true_nn(path: str, ids: np.ndarray, dists: np.ndarray) -> None:
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    dists = np.ascontiguousarray(dists, dtype=np.float32)
    nq, k = ids.shape
    body = np.empty((nq, k, 2), dtype=np.uint32)
    body[:, :, 0] = ids
    body[:, :, 1] = dists.view(np.uint32)
    with open(path, "wb") as f:
        np.array([nq, k], dtype=np.uint32).tofile(f)
        body.tofile(f)


def read_true_nn(path: str):
    raw = np.fromfile(path, dtype=np.uint32)
    nq, k = int(raw[0]), int(raw[1])
    body = raw[2:2 + nq * k * 2].reshape(nq, k, 2)
    return body[:, :, 0].copy(), body[:, :, 1].copy().view(np.float32)


def write_results(path: str, ids: np.ndarray) -> None:
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    nq, k = ids.shape
    rec = np.empty((nq, k + 1), dtype=np.uint32)
    rec[:, 0] = k
    rec[:, 1:] = ids
    rec.tofile(path)


def read_results(path: str) -> np.ndarray:
    raw = np.fromfile(path, dtype=np.uint32)
    if raw.size == 0:
        return np.zeros((0, 0), dtype=np.uint32)
    k = int(raw[0])
    return raw.reshape(-1, k + 1)[:, 1:].copy()


def file_size(path: str) -> int:
    return os.stat(path).st_size
