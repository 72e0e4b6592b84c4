"""ctypes wrapper of the CPU oracle (oracle/_ref/panns_oracle.so) and of the
reference binaries (oracle/_ref/ref_*) — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module, and only to check results. The product never does.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
SO_PATH = os.path.join(REF_DIR, "panns_oracle.so")

DIST_IP_NORM = 0
DIST_L2 = 1

_lib = None


def build(ref_root: str | None = None) -> None:
    """Build the C oracle, and the reference binaries when the
    reference sources are present."""
    targets = ["oracle"]
    env = dict(os.environ)
    if ref_root and os.path.isdir(ref_root):
        targets = ["all"]
    args = ["make", "-s", "-C", HERE] + targets
    if ref_root:
        args.append(f"REF={ref_root}")
    subprocess.run(args, check=True, env=env)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SO_PATH):
            build()
        L = ctypes.CDLL(SO_PATH)
        P = ctypes.c_void_p
        u32 = ctypes.c_uint32
        L.po_norm.restype = ctypes.c_float
        L.po_norm.argtypes = [P, ctypes.c_int, ctypes.c_int]
        L.po_distance.restype = ctypes.c_float
        L.po_distance.argtypes = [P, P, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.po_set_fused.argtypes = [ctypes.c_int]
        L.po_prepare_init_ids.argtypes = [P, P, u32, u32, u32, P]
        L.po_rand_state_size.restype = u32
        L.po_srand.argtypes = [P, u32]
        L.po_rand.restype = ctypes.c_int32
        L.po_rand.argtypes = [P]
        L.po_efanna_init_ids.argtypes = [P, P, u32, u32, u32, u32, P, P]
        L.po_search_top_m.argtypes = [P, P, u32, u32, P, P, P, u32, P, ctypes.c_int, u32, u32, u32,
                                      ctypes.c_int, P, P, ctypes.c_int]
        L.po_search_top_m_lists.argtypes = [P, P, u32, u32, P, P, P, u32, P, u32, P, P, u32, u32,
                                            ctypes.c_int, P, P, ctypes.c_int]
        L.po_build_nsg.argtypes = [P, u32, u32, u32, u32, P, P, P, P, ctypes.c_uint64, P, ctypes.c_int]
        L.po_search_pss.argtypes = [P, P, u32, u32, P, P, P, u32, P, u32, u32, u32, u32, u32,
                                    ctypes.c_int, P, P, ctypes.c_int]
        L.po_search_efanna.argtypes = [P, P, u32, u32, P, P, P, u32, P, u32, u32, ctypes.c_int,
                                       P, P, ctypes.c_int]
        L.po_ground_truth_fp64.argtypes = [P, u32, u32, P, u32, u32, P, P, ctypes.c_int]
        L.po_host_knn.argtypes = [P, u32, u32, P, u32, u32, P, P, ctypes.c_int]
        L.po_host_build_nsg.argtypes = [P, u32, u32, u32, u32, P, P, P, P, ctypes.c_uint64, P, ctypes.c_int]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _threads(t):
    return t if t else (os.cpu_count() or 1)


class Graph:
    """CSR view used by the oracle: offsets (u64, N+1), nbrs (u32)."""

    def __init__(self, offsets, nbrs, entry, width=None):
        self.offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        self.nbrs = np.ascontiguousarray(nbrs, dtype=np.uint32)
        self.entry = int(entry)
        self.n = self.offsets.shape[0] - 1
        self.width = width

    @staticmethod
    def from_nsg(g):
        return Graph(g.offsets, g.nbrs, g.entry, g.width)


def norms(data: np.ndarray, fused: int = 1) -> np.ndarray:
    """||v||^2 per row in the reference's lane order (FMA lane steps by
    default, as the reference's -march=native build computes it)."""
    L = lib()
    data = np.ascontiguousarray(data, dtype=np.float32)
    d = data.shape[1]
    out = np.empty(data.shape[0], dtype=np.float32)
    for i in range(data.shape[0]):
        out[i] = L.po_norm(data[i].ctypes.data_as(ctypes.c_void_p), d, fused)
    return out


def distance(v, q, norm, kind, fused=1) -> float:
    v = np.ascontiguousarray(v, dtype=np.float32)
    q = np.ascontiguousarray(q, dtype=np.float32)
    return float(lib().po_distance(_p(v), _p(q), ctypes.c_float(norm), v.shape[0], kind, fused))


def prepare_init_ids(g: Graph, L: int) -> np.ndarray:
    out = np.empty(L, dtype=np.uint32)
    rc = lib().po_prepare_init_ids(_p(g.offsets), _p(g.nbrs), g.n, g.entry, L, _p(out))
    if rc:
        raise ValueError(f"po_prepare_init_ids failed ({rc})")
    return out


class Rand:
    """glibc rand() stream, independent of the process-wide one."""

    def __init__(self, seed: int = 1):
        self.buf = ctypes.create_string_buffer(lib().po_rand_state_size())
        lib().po_srand(self.buf, seed)

    def __call__(self) -> int:
        return int(lib().po_rand(self.buf))


def efanna_init_ids(g: Graph, L: int, nq: int, rng: Rand | None = None) -> np.ndarray:
    rng = rng or Rand(1)
    out = np.empty((nq, L), dtype=np.uint32)
    rc = lib().po_efanna_init_ids(_p(g.offsets), _p(g.nbrs), g.n, g.entry, L, nq, rng.buf, _p(out))
    if rc:
        raise ValueError(f"po_efanna_init_ids failed ({rc})")
    return out


def _vec_args(data, queries):
    data = np.ascontiguousarray(data, dtype=np.float32)
    queries = np.ascontiguousarray(queries, dtype=np.float32)
    return data, queries


def search_top_m(data, g: Graph, queries, K, L, M=1, kind=DIST_IP_NORM, init_ids=None,
                 nrm=None, threads=0):
    data, queries = _vec_args(data, queries)
    n, d = data.shape
    nq = queries.shape[0]
    if init_ids is None:
        init_ids = prepare_init_ids(g, L)
    init_ids = np.ascontiguousarray(init_ids, dtype=np.uint32)
    per_q = 1 if init_ids.ndim == 2 else 0
    if kind == DIST_IP_NORM and nrm is None:
        nrm = norms(data)
    nrm_p = _p(nrm) if kind == DIST_IP_NORM else None
    out = np.empty((nq, K), dtype=np.uint32)
    nd = np.zeros(1, dtype=np.uint64)
    rc = lib().po_search_top_m(_p(data), nrm_p, n, d, _p(g.offsets), _p(g.nbrs), _p(queries), nq,
                               _p(init_ids), per_q, K, L, M, kind, _p(out), _p(nd),
                               _threads(threads))
    if rc:
        raise ValueError(f"po_search_top_m failed ({rc})")
    return out, int(nd[0])


def search_top_m_lists(data, g: Graph, queries, K, Lq, M, init_lists, kind=DIST_IP_NORM, nrm=None,
                       threads=0):
    """Top-M search where query i starts from init_lists[i] (any length <=
    Lq[i]; repeated ids enter once) with its own queue length Lq[i]."""
    data, queries = _vec_args(data, queries)
    n, d = data.shape
    nq = queries.shape[0]
    Lq = np.ascontiguousarray(Lq, dtype=np.uint32)
    stride = max(1, max(len(x) for x in init_lists))
    lists = np.zeros((nq, stride), dtype=np.uint32)
    counts = np.zeros(nq, dtype=np.uint32)
    for i, x in enumerate(init_lists):
        lists[i, :len(x)] = x
        counts[i] = len(x)
    if kind == DIST_IP_NORM and nrm is None:
        nrm = norms(data)
    nrm_p = _p(nrm) if kind == DIST_IP_NORM else None
    out = np.empty((nq, K), dtype=np.uint32)
    nd = np.zeros(1, dtype=np.uint64)
    rc = lib().po_search_top_m_lists(_p(data), nrm_p, n, d, _p(g.offsets), _p(g.nbrs), _p(queries), nq,
                                     _p(lists), stride, _p(counts), _p(Lq), K, M, kind, _p(out), _p(nd),
                                     _threads(threads))
    if rc:
        raise ValueError(f"po_search_top_m_lists failed ({rc})")
    return out, int(nd[0])


def search_pss(data, g: Graph, queries, K, L, L_local=None, X=1, T=1, kind=DIST_IP_NORM,
               init_ids=None, nrm=None, threads=0):
    data, queries = _vec_args(data, queries)
    n, d = data.shape
    nq = queries.shape[0]
    L_local = L if L_local is None else L_local
    if init_ids is None:
        init_ids = prepare_init_ids(g, L)
    init_ids = np.ascontiguousarray(init_ids, dtype=np.uint32)
    if kind == DIST_IP_NORM and nrm is None:
        nrm = norms(data)
    nrm_p = _p(nrm) if kind == DIST_IP_NORM else None
    out = np.empty((nq, K), dtype=np.uint32)
    nd = np.zeros(1, dtype=np.uint64)
    rc = lib().po_search_pss(_p(data), nrm_p, n, d, _p(g.offsets), _p(g.nbrs), _p(queries), nq,
                             _p(init_ids), K, L, L_local, X, T, kind, _p(out), _p(nd),
                             _threads(threads))
    if rc:
        raise ValueError(f"po_search_pss failed ({rc})")
    return out, int(nd[0])


def search_efanna(data, g: Graph, queries, K, L, kind=DIST_L2, init_ids=None, nrm=None,
                  threads=0):
    data, queries = _vec_args(data, queries)
    n, d = data.shape
    nq = queries.shape[0]
    if init_ids is None:
        init_ids = efanna_init_ids(g, L, nq)
    init_ids = np.ascontiguousarray(init_ids, dtype=np.uint32)
    if kind == DIST_IP_NORM and nrm is None:
        nrm = norms(data)
    nrm_p = _p(nrm) if kind == DIST_IP_NORM else None
    out = np.empty((nq, K), dtype=np.uint32)
    nd = np.zeros(1, dtype=np.uint64)
    rc = lib().po_search_efanna(_p(data), nrm_p, n, d, _p(g.offsets), _p(g.nbrs), _p(queries), nq,
                                _p(init_ids), K, L, kind, _p(out), _p(nd), _threads(threads))
    if rc:
        raise ValueError(f"po_search_efanna failed ({rc})")
    return out, int(nd[0])


def ground_truth(data, queries, k=100, threads=0):
    data, queries = _vec_args(data, queries)
    n, d = data.shape
    nq = queries.shape[0]
    ids = np.empty((nq, k), dtype=np.uint32)
    dist = np.empty((nq, k), dtype=np.float64)
    rc = lib().po_ground_truth_fp64(_p(data), n, d, _p(queries), nq, k, _p(ids), _p(dist),
                                    _threads(threads))
    if rc:
        raise ValueError(f"po_ground_truth_fp64 failed ({rc})")
    return ids, dist


def recall_at(result_ids: np.ndarray, true_ids: np.ndarray, L: int, at: int = 100) -> float:
    """The reference's recall definition
    (core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp:191-230):
    hits of the true top-`at` within result[0:min(L, 100)] prefix `at`."""
    kk = min(L, 100, result_ids.shape[1])
    res = result_ids[:, :min(kk, at)]
    tru = true_ids[:, :at]
    hits = 0
    for r, t in zip(res, tru):
        hits += np.intersect1d(r, t).size
    return hits / float(at * result_ids.shape[0])


# --- reference binaries -------------------------------------------

def ref_binary(name: str) -> str:
    return os.path.join(REF_DIR, name)


def ref_nsg_build(base_path: str, knn_path: str, L: int, R: int, C: int, out_path: str, threads: int = 1):
    """efanna2e IndexNSG::Build by the reference's tools/test_nsg_index.cpp
    (oracle/_ref/ref_nsg_build) at `threads` OpenMP threads."""
    args = [ref_binary("ref_nsg_build"), base_path, knn_path, str(L), str(R), str(C), out_path, str(threads)]
    r = subprocess.run(args, check=True, capture_output=True, text=True)
    return r.stdout


def write_efanna_knn(path: str, knn: np.ndarray) -> None:
    """An EFANNA k-NN graph file (what IndexNSG::Load_nn_graph reads): per
    vertex u32 k, then k u32 ids."""
    knn = np.ascontiguousarray(knn, dtype=np.uint32)
    rec = np.empty((knn.shape[0], knn.shape[1] + 1), dtype=np.uint32)
    rec[:, 0] = knn.shape[1]
    rec[:, 1:] = knn
    rec.tofile(path)


def read_efanna_knn(path: str) -> np.ndarray:
    raw = np.fromfile(path, dtype=np.uint32)
    k = int(raw[0])
    return raw.reshape(-1, k + 1)[:, 1:].copy()


def have_ref() -> bool:
    return all(os.path.exists(ref_binary(b)) for b in ("ref_pss", "ref_pss_lg", "ref_topm", "ref_efanna"))


def run_ref(name: str, out_path: str, env=None, **kw):
    """Run a reference binary; returns (ids [nq x K], stats dict)."""
    args = [ref_binary(name)] + [f"{k}={v}" for k, v in kw.items()] + [f"out={out_path}"]
    r = subprocess.run(args, check=True, capture_output=True, text=True, env=env)
    stats = json.loads(r.stdout.strip().splitlines()[-1]) if r.stdout.strip() else {}
    if kw.get("mode") == "dist":
        return None, stats
    K = int(kw.get("K", 100))
    ids = np.fromfile(out_path, dtype=np.uint32).reshape(-1, K)
    return ids, stats


def build_nsg(base, k, R, threads=0):
    """The graph construction restated in C: returns (NSGGraph, knn ids n x k)."""
    from parallel_anns_b200.formats import NSGGraph
    x = np.ascontiguousarray(base, dtype=np.float32)
    n, d = x.shape
    knn = np.empty((n, k), dtype=np.uint32)
    off = np.empty(n + 1, dtype=np.uint64)
    cap = n * R + n  # repair adds at most one in-edge per vertex
    nbrs = np.empty(cap, dtype=np.uint32)
    entry = np.zeros(1, dtype=np.uint32)
    width = np.zeros(1, dtype=np.uint32)
    rc = lib().po_build_nsg(_p(x), n, d, k, R, _p(knn), _p(entry), _p(off), _p(nbrs), cap, _p(width),
                            _threads(threads))
    if rc:
        raise ValueError(f"po_build_nsg failed ({rc})")
    g = NSGGraph(int(width[0]), int(entry[0]), off.astype(np.int64), nbrs[:int(off[-1])].copy())
    return g, knn


def host_knn(base, queries, k, threads=0):
    """Exact top-k by (float64 FMA-chain distance, id) with cluster lower
    bounds (oracle/host_build.c); queries=None: the k-NN of every base row,
    itself excluded. Returns (ids u32 [nq x k], float64 distances)."""
    x = np.ascontiguousarray(base, dtype=np.float32)
    n, d = x.shape
    if queries is None:
        qp, nq = None, n
    else:
        queries = np.ascontiguousarray(queries, dtype=np.float32)
        qp, nq = _p(queries), queries.shape[0]
    ids = np.empty((nq, k), dtype=np.uint32)
    dist = np.empty((nq, k), dtype=np.float64)
    rc = lib().po_host_knn(_p(x), n, d, qp, nq if queries is not None else 0, k, _p(ids), _p(dist),
                           _threads(threads))
    if rc:
        raise ValueError(f"po_host_knn failed ({rc})")
    return ids, dist


def host_build_nsg(base, k, R, threads=0):
    """po_build_nsg's graph, built with cluster lower bounds (seconds at 1M):
    returns (NSGGraph, knn ids n x k)."""
    from parallel_anns_b200.formats import NSGGraph
    x = np.ascontiguousarray(base, dtype=np.float32)
    n, d = x.shape
    knn = np.empty((n, k), dtype=np.uint32)
    off = np.empty(n + 1, dtype=np.uint64)
    cap = n * R + n
    nbrs = np.empty(cap, dtype=np.uint32)
    entry = np.zeros(1, dtype=np.uint32)
    width = np.zeros(1, dtype=np.uint32)
    rc = lib().po_host_build_nsg(_p(x), n, d, k, R, _p(knn), _p(entry), _p(off), _p(nbrs), cap, _p(width),
                                 _threads(threads))
    if rc:
        raise ValueError(f"po_host_build_nsg failed ({rc})")
    g = NSGGraph(int(width[0]), int(entry[0]), off.astype(np.int64), nbrs[:int(off[-1])].copy())
    return g, knn
