"""GPU graph construction (include/panns_build.h): exact k-NN, MRNG prune to
R, medoid entry, reachability repair — the NSG-style graphs the benchmark
workloads describe, built by the library's own kernels."""
from __future__ import annotations

import ctypes

import numpy as np

from . import native as N
from .formats import NSGGraph


SCREEN_AUTO, SCREEN_FP32, SCREEN_TF32, SCREEN_TC = 0, 1, 2, 3


def build_nsg(base: np.ndarray, R: int = 50, knn_k: int = 64, device: int = 0, with_knn: bool = False,
              screen: int = SCREEN_AUTO):
    """Build the graph of ``base`` (n x d float32) on GPU ``device``.
    Returns an NSGGraph (and the n x knn_k k-NN ids if ``with_knn``)."""
    x = np.ascontiguousarray(base, dtype=np.float32)
    n, d = x.shape
    lib = N.load()
    g = ctypes.c_void_p()
    N.check(lib.panns_build_nsg_ex(device, N.ptr(x), n, d, knn_k, R, screen, ctypes.byref(g)))
    try:
        vals = [ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint32()]
        N.check(lib.panns_graph_info(g, *[ctypes.byref(v) for v in vals]))
        _, width, entry, n_edges, repaired = [v.value for v in vals]
        off = np.empty(n + 1, dtype=np.uint64)
        nbrs = np.empty(max(n_edges, 1), dtype=np.uint32)
        knn = np.empty((n, knn_k), dtype=np.uint32) if with_knn else None
        N.check(lib.panns_graph_copy(g, N.ptr(off), N.ptr(nbrs), N.ptr(knn) if with_knn else None))
    finally:
        lib.panns_graph_free(g)
    graph = NSGGraph(int(width), int(entry), off.astype(np.int64), nbrs[:n_edges].copy())
    graph.repaired = repaired
    return (graph, knn) if with_knn else graph


def build_nsg_cells(base: np.ndarray, R: int = 48, knn_k: int = 64, cells: int = 10_000, probe: int = 3,
                    sample: int = 2_000_000, iters: int = 10, seed: int = 1, device: int = 0,
                    reverse: bool = False, with_knn: bool = False, with_cells: bool = False):
    """The large-graph construction (include/panns_build.h, panns_build_nsg_cells):
    k-NN lists among each vertex's k-means cell and its ``probe`` nearest
    cells, then the same prune, entry and repair as ``build_nsg`` (with
    ``reverse``, reverse edges up to R before the repair). Returns an
    NSGGraph, plus the k-NN ids if ``with_knn`` and (cell of every vertex,
    cells x probe nearest cells) if ``with_cells``."""
    x = np.ascontiguousarray(base, dtype=np.float32)
    n, d = x.shape
    lib = N.load()
    g = ctypes.c_void_p()
    N.check(lib.panns_build_nsg_cells(device, N.ptr(x), n, d, knn_k, R, cells, probe, sample, iters, seed,
                                      int(bool(reverse)), ctypes.byref(g)))
    try:
        vals = [ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint32()]
        N.check(lib.panns_graph_info(g, *[ctypes.byref(v) for v in vals]))
        _, width, entry, n_edges, repaired = [v.value for v in vals]
        off = np.empty(n + 1, dtype=np.uint64)
        nbrs = np.empty(max(n_edges, 1), dtype=np.uint32)
        knn = np.empty((n, knn_k), dtype=np.uint32) if with_knn else None
        N.check(lib.panns_graph_copy(g, N.ptr(off), N.ptr(nbrs), N.ptr(knn) if with_knn else None))
        part = None
        if with_cells:
            nc, npb = ctypes.c_uint32(), ctypes.c_uint32()
            N.check(lib.panns_graph_cells(g, ctypes.byref(nc), ctypes.byref(npb), None, None))
            cell = np.empty(n, dtype=np.uint32)
            near = np.empty((nc.value, max(npb.value, 1)), dtype=np.uint32)
            N.check(lib.panns_graph_cells(g, None, None, N.ptr(cell), N.ptr(near)))
            part = (cell, near[:, :npb.value])
    finally:
        lib.panns_graph_free(g)
    graph = NSGGraph(int(width), int(entry), off.astype(np.int64), nbrs[:n_edges].copy())
    graph.repaired = repaired
    out = [graph]
    if with_knn:
        out.append(knn)
    if with_cells:
        out.append(part)
    return out[0] if len(out) == 1 else tuple(out)


def save_nsg_gpu_built(base: np.ndarray, path: str, R: int = 50, knn_k: int = 64, device: int = 0) -> None:
    """Build and write the .nsg file directly from the library (IndexNSG::Save layout)."""
    x = np.ascontiguousarray(base, dtype=np.float32)
    lib = N.load()
    g = ctypes.c_void_p()
    N.check(lib.panns_build_nsg(device, N.ptr(x), x.shape[0], x.shape[1], knn_k, R, ctypes.byref(g)))
    try:
        N.check(lib.panns_graph_save_nsg(g, path.encode()))
    finally:
        lib.panns_graph_free(g)


def efanna_build(base: np.ndarray, knn: np.ndarray, L: int, R: int, C: int, rand_seed: int = 1,
                 device: int = 0) -> NSGGraph:
    """efanna2e's IndexNSG::Build from a k-NN graph (n x k ids), the result
    equal to the reference's at one thread (include/panns_build.h)."""
    x = np.ascontiguousarray(base, dtype=np.float32)
    kn = np.ascontiguousarray(knn, dtype=np.uint32)
    n, d = x.shape
    lib = N.load()
    g = ctypes.c_void_p()
    N.check(lib.panns_efanna_build(device, N.ptr(x), n, d, N.ptr(kn), kn.shape[1], L, R, C, rand_seed,
                                   ctypes.byref(g)))
    try:
        vals = [ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint32()]
        N.check(lib.panns_graph_info(g, *[ctypes.byref(v) for v in vals]))
        _, width, entry, n_edges, _ = [v.value for v in vals]
        off = np.empty(n + 1, dtype=np.uint64)
        nbrs = np.empty(max(n_edges, 1), dtype=np.uint32)
        N.check(lib.panns_graph_copy(g, N.ptr(off), N.ptr(nbrs), None))
    finally:
        lib.panns_graph_free(g)
    return NSGGraph(int(width), int(entry), off.astype(np.int64), nbrs[:n_edges].copy())
