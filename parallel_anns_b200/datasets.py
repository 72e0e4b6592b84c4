"""Synthetic inputs and NSG-style graph construction for the search path.

The reference measures on SIFT/GIST/DEEP files that are not available here.
These seeded generators stand in for them with the shapes of the workloads the
search is benchmarked on: an isotropic Gaussian mixture (component means drawn
from N(0, 1), per-coordinate sigma), every vector L2-normalised to unit norm.

Graph construction (``build_nsg_graph``) follows a simple NSG recipe:

1. exact k-NN lists (default 64) by brute force, ordered by (distance, id);
2. relative-neighbourhood (MRNG) pruning: walking a vertex's list in order, a
   candidate b is dropped when an already-kept neighbour c has d(b, c) < d(a, b);
   at most R neighbours are kept (the occlusion rule of
   ``include/efanna2e/index_nsg.cpp:233-283`` ``sync_prune``, applied to the exact
   k-NN list instead of a search pool);
3. entry vertex = medoid, the vertex nearest to the centroid;
4. reachability repair from the entry (the role of ``tree_grow`` / ``DFS`` /
   ``findroot`` in ``include/efanna2e/index_nsg.cpp:638-718``): every vertex not
   reachable from the entry gets an in-edge from the first reachable vertex of
   its own k-NN list (the entry if none is reachable), in increasing id order,
   and everything it reaches is marked reachable before the next one.

``width`` of the written graph is its maximum out-degree after repair.

The brute-force steps run with torch on the given device (CUDA GEMMs on the GPU
host, CPU otherwise); they prepare inputs and are not part of the search path.
"""
from __future__ import annotations

from collections import deque

import numpy as np
import torch

from .formats import NSGGraph


def gaussian_mixture(n: int, d: int, n_components: int = 64, sigma: float = 0.3,
                     seed: int = 0, means_seed: int | None = None,
                     normalize: bool = True) -> np.ndarray:
    """``n`` float32 vectors from an isotropic Gaussian mixture.

    The component means come from ``means_seed`` (default ``seed``), so base
    vectors and queries drawn with different ``seed`` but the same
    ``means_seed`` share one mixture.
    """
    mrng = np.random.default_rng(seed if means_seed is None else means_seed)
    means = mrng.standard_normal((n_components, d), dtype=np.float32)
    rng = np.random.default_rng(seed + 0x9E3779B9)
    comp = rng.integers(0, n_components, size=n)
    x = rng.standard_normal((n, d), dtype=np.float32)
    x *= np.float32(sigma)
    x += means[comp]
    if normalize:
        nrm = np.sqrt(np.einsum("ij,ij->i", x.astype(np.float64), x.astype(np.float64)))
        nrm[nrm == 0] = 1.0
        x = (x / nrm[:, None]).astype(np.float32)
    return np.ascontiguousarray(x, dtype=np.float32)


@torch.no_grad()
def gaussian_mixture_gpu(n: int, d: int, n_components: int = 4096, sigma: float = 0.3, seed: int = 0,
                         means_seed: int | None = None, chunk: int = 1 << 20, device: int = 0) -> np.ndarray:
    """``n`` float32 vectors from the same kind of mixture as ``gaussian_mixture``
    (means ~ N(0, 1), per-coordinate sigma, unit norm), drawn on the GPU with
    torch's seeded Philox generator, chunk by chunk into host memory, for
    bases too large for host-side float64 temporaries (100M x 96). The means
    come from ``means_seed`` (default ``seed``); chunk i uses the stream of
    (seed, i), so the result does not depend on memory size."""
    dev = torch.device("cuda", device)
    gm = torch.Generator(device=dev)
    gm.manual_seed(seed if means_seed is None else means_seed)
    means = torch.randn((n_components, d), generator=gm, device=dev, dtype=torch.float32)
    out = np.empty((n, d), dtype=np.float32)
    pinned = torch.empty((min(chunk, n), d), dtype=torch.float32).pin_memory()
    g = torch.Generator(device=dev)
    for i, r0 in enumerate(range(0, n, chunk)):
        m = min(chunk, n - r0)
        g.manual_seed((seed * 1_000_003 + i) & 0x7FFFFFFFFFFFFFFF)
        comp = torch.randint(0, n_components, (m,), generator=g, device=dev)
        x = torch.randn((m, d), generator=g, device=dev, dtype=torch.float32) * sigma + means[comp]
        nrm = torch.linalg.vector_norm(x.double(), dim=1, keepdim=True)
        nrm[nrm == 0] = 1.0
        x = (x.double() / nrm).float()
        pinned[:m].copy_(x)
        out[r0:r0 + m] = pinned[:m].numpy()
    return out


def uint8_cube(n: int, d: int = 128, seed: int = 0) -> np.ndarray:
    """Integer-valued components uniform in 0..255, stored as uint8 then cast."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, 256, size=(n, d), dtype=np.uint8).astype(np.float32)


def _device(device) -> torch.device:
    if device is None:
        return torch.device("cuda" if torch.cuda.is_available() else "cpu")
    return torch.device(device)


@torch.no_grad()
def exact_knn(base: np.ndarray, queries: np.ndarray, k: int, exclude_self: bool = False,
              device=None, block: int = 4096, dtype=torch.float32):
    """Exact k nearest neighbours by brute force, ordered by (distance, id).

    Distances are squared L2 computed as ||x||^2 + ||q||^2 - 2 x.q in ``dtype``;
    the returned distances are recomputed exactly as sum((x - q)^2) in float64
    for the selected ids and the final order is by that float64 distance, then id.
    """
    dev = _device(device)
    xb = torch.from_numpy(np.ascontiguousarray(base)).to(dev, dtype)
    nb = xb.shape[0]
    xn = (xb.double() * xb.double()).sum(1).to(dtype)
    kk = min(k + (1 if exclude_self else 0) + 8, nb)
    out_ids = np.empty((queries.shape[0], k), dtype=np.uint32)
    out_d = np.empty((queries.shape[0], k), dtype=np.float64)
    prev_tf32 = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for s in range(0, queries.shape[0], block):
            q = torch.from_numpy(np.ascontiguousarray(queries[s:s + block])).to(dev, dtype)
            qn = (q.double() * q.double()).sum(1).to(dtype)
            dist = qn[:, None] + xn[None, :] - 2.0 * (q @ xb.T)
            if exclude_self:
                rows = torch.arange(q.shape[0], device=dev)
                dist[rows, rows + s] = float("inf")
            cand = torch.topk(dist, kk, dim=1, largest=False).indices
            # Exact float64 re-rank of the shortlist, then (distance, id) order.
            diff = xb[cand].double() - q[:, None, :].double()
            d64 = (diff * diff).sum(-1)
            if exclude_self:
                d64[cand == (torch.arange(q.shape[0], device=dev)[:, None] + s)] = float("inf")
            key_order = torch.argsort(cand, dim=1, stable=True)
            cand = torch.gather(cand, 1, key_order)
            d64 = torch.gather(d64, 1, key_order)
            order = torch.argsort(d64, dim=1, stable=True)[:, :k]
            out_ids[s:s + q.shape[0]] = torch.gather(cand, 1, order).cpu().numpy().astype(np.uint32)
            out_d[s:s + q.shape[0]] = torch.gather(d64, 1, order).cpu().numpy()
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev_tf32
    return out_ids, out_d


@torch.no_grad()
def mrng_prune(base: np.ndarray, knn_ids: np.ndarray, knn_d: np.ndarray, R: int,
               device=None, block: int = 8192) -> list:
    """Relative-neighbourhood pruning of exact k-NN lists to at most R neighbours."""
    dev = _device(device)
    xb = torch.from_numpy(np.ascontiguousarray(base)).to(dev, torch.float64)
    n, k = knn_ids.shape
    lists = []
    for s in range(0, n, block):
        ids = torch.from_numpy(knn_ids[s:s + block].astype(np.int64)).to(dev)
        dab = torch.from_numpy(knn_d[s:s + block]).to(dev)
        v = xb[ids]  # [b, k, d]
        gram = v @ v.transpose(1, 2)
        sq = torch.diagonal(gram, dim1=1, dim2=2)
        pd = sq[:, :, None] + sq[:, None, :] - 2 * gram  # d(c, b) for c, b in the list
        b = ids.shape[0]
        keep = torch.zeros((b, k), dtype=torch.bool, device=dev)
        kept = torch.zeros(b, dtype=torch.int64, device=dev)
        for i in range(k):
            # occluded if some kept c (j < i) has d(c, b_i) < d(a, b_i)
            occl = (keep[:, :i] & (pd[:, :i, i] < dab[:, i:i + 1])).any(1) if i else \
                torch.zeros(b, dtype=torch.bool, device=dev)
            ok = (~occl) & (kept < R)
            keep[:, i] = ok
            kept += ok.long()
        keep_np = keep.cpu().numpy()
        ids_np = knn_ids[s:s + block]
        cnt = keep_np.sum(1)
        flat = ids_np[keep_np].astype(np.uint32)  # row-major: each row's kept ids in order
        lists.extend(np.split(flat, np.cumsum(cnt)[:-1]))
    return lists


def medoid(base: np.ndarray) -> int:
    c = base.astype(np.float64).mean(0)
    d = ((base.astype(np.float64) - c) ** 2).sum(1)
    return int(np.argmin(d))


def _reached_from(lists: list, src: int, n: int) -> np.ndarray:
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import breadth_first_order
    deg = np.array([len(l) for l in lists], dtype=np.int64)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(deg, out=indptr[1:])
    idx = np.concatenate(lists).astype(np.int64) if indptr[-1] else np.zeros(0, np.int64)
    m = csr_matrix((np.ones(idx.shape[0], dtype=np.int8), idx, indptr), shape=(n, n))
    order = breadth_first_order(m, src, directed=True, return_predecessors=False)
    reached = np.zeros(n, dtype=bool)
    reached[order] = True
    return reached


def repair_reachability(lists: list, entry: int, knn_ids: np.ndarray) -> int:
    """Give every vertex unreachable from ``entry`` an in-edge; returns edges added."""
    n = len(lists)
    reached = _reached_from(lists, entry, n)
    added = 0
    for u in np.nonzero(~reached)[0]:
        u = int(u)
        if reached[u]:
            continue
        parent = entry
        for c in knn_ids[u]:
            if reached[c]:
                parent = int(c)
                break
        lists[parent] = np.append(lists[parent], np.uint32(u))
        added += 1
        # mark everything u reaches (only not-yet-reached vertices are walked)
        dq = deque([u])
        reached[u] = True
        while dq:
            x = dq.popleft()
            for w in lists[x]:
                if not reached[w]:
                    reached[w] = True
                    dq.append(int(w))
    return added


def build_nsg_graph(base: np.ndarray, R: int = 50, knn_k: int = 64, device=None,
                    knn=None) -> NSGGraph:
    """NSG-style graph: exact k-NN, MRNG prune to R, medoid entry, reachability repair."""
    if knn is None:
        knn = exact_knn(base, base, knn_k, exclude_self=True, device=device)
    knn_ids, knn_d = knn
    lists = mrng_prune(base, knn_ids, knn_d, R, device=device)
    entry = medoid(base)
    repair_reachability(lists, entry, knn_ids)
    width = max(len(l) for l in lists)
    return NSGGraph.from_lists(width, entry, lists)


def ground_truth_fp64_cpu(base: np.ndarray, queries: np.ndarray, k: int = 100):
    """Top-k by exact float64 squared L2, ties by id (CPU; small inputs only)."""
    ids, d = exact_knn(base, queries, k, device="cpu", dtype=torch.float64)
    return ids, d.astype(np.float32)
