"""Host-side mirror of the reference's search interfaces over the C ABI.

* ``Index`` — the batched engine: one GPU handle holding base vectors, graph
  and queries; ``search`` runs many queries in one launch.
* ``Searching`` — the method names, argument meanings and call pattern of
  ``PANNS::Searching`` (core/Searching.202102022027.PSS_v5.dist_thresh.profiling.h:30-274,
  core/Searching.202102031939.PSS_v5.large_graph.dist_thresh.profiling.h,
  core/Searching.202011241533.top_m_pure.h): loaders, ``prepare_init_ids``,
  the per-query search methods writing ``set_K``, ``load_true_NN`` and
  ``get_recall_for_all_queries``; plus ``*_batch`` forms that fill a whole
  ``set_K_list`` in one GPU launch.
* ``IndexNSG`` — efanna2e::IndexNSG's query path (include/efanna2e/index_nsg.h:17-43):
  ``Load``, ``OptimizeGraph``, ``Search``, ``SearchWithOptGraph``, with the
  process-wide ``rand()`` stream of the reference replayed per query.

Errors raise ``PannsError`` (the reference calls exit(EXIT_FAILURE)).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import native as N
from .formats import NSGGraph, read_true_nn


class Index:
    """A GPU-resident base set + NSG graph (+ optional loaded queries)."""

    def __init__(self, device: int = 0):
        self._lib = N.load()
        h = ctypes.c_void_p()
        N.check(self._lib.panns_open(ctypes.byref(h), int(device)))
        self._h = h
        self.n = 0
        self.d = 0
        self.nq = 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.panns_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- loaders ----------------------------------------------------------
    def set_base(self, data: np.ndarray, storage: int = N.STORE_FP32):
        data = np.ascontiguousarray(data, dtype=np.float32)
        N.check(self._lib.panns_set_base(self._h, N.ptr(data), data.shape[0], data.shape[1], storage))
        self.n, self.d = data.shape

    def load_fvecs_base(self, path: str, storage: int = N.STORE_FP32):
        N.check(self._lib.panns_load_fvecs_base(self._h, path.encode(), storage))
        self._refresh()

    def set_queries(self, queries: np.ndarray):
        queries = np.ascontiguousarray(queries, dtype=np.float32)
        N.check(self._lib.panns_set_queries(self._h, N.ptr(queries), queries.shape[0],
                                            queries.shape[1]))
        self.nq = queries.shape[0]

    def load_fvecs_queries(self, path: str):
        N.check(self._lib.panns_load_fvecs_queries(self._h, path.encode()))
        self._refresh()

    def set_graph(self, g: NSGGraph):
        off = np.ascontiguousarray(g.offsets, dtype=np.uint64)
        nb = np.ascontiguousarray(g.nbrs, dtype=np.uint32)
        N.check(self._lib.panns_set_graph(self._h, int(g.width), int(g.entry), N.ptr(off),
                                          N.ptr(nb) if nb.size else None, g.n))

    def load_nsg(self, path: str):
        N.check(self._lib.panns_load_nsg(self._h, path.encode()))
        self._refresh()

    def info(self):
        vals = [ctypes.c_uint32() for _ in range(5)]
        N.check(self._lib.panns_info(self._h, *[ctypes.byref(v) for v in vals]))
        return dict(zip(("n", "d", "nq", "width", "entry"), [v.value for v in vals]))

    def _refresh(self):
        i = self.info()
        self.n, self.d, self.nq = i["n"], i["d"], i["nq"]

    # -- init ids -----------------------------------------------------------
    def prepare_init_ids(self, L: int) -> np.ndarray:
        out = np.empty(L, dtype=np.uint32)
        N.check(self._lib.panns_prepare_init_ids(self._h, L, N.ptr(out)))
        return out

    @staticmethod
    def rand_state(seed: int = 1) -> np.ndarray:
        st = np.zeros(40, dtype=np.int32)
        N.check(N.load().panns_rand_seed(N.ptr(st), seed))
        return st

    def efanna_init_ids(self, L: int, nq: int, rand_state: np.ndarray | None = None) -> np.ndarray:
        st = self.rand_state(1) if rand_state is None else rand_state
        out = np.empty((nq, L), dtype=np.uint32)
        N.check(self._lib.panns_efanna_init_ids(self._h, L, nq, N.ptr(st), N.ptr(out)))
        return out

    # -- search ---------------------------------------------------------------
    @staticmethod
    def params(mode=N.MODE_NSG_SEQ, distance=N.DIST_NORM_IP, K=100, L=100, M=1, T=1,
               L_local=0, X=1, warps_per_block=0, storage=N.STORE_FP32, flags=0,
               L_query=None, blocks_per_sm=0, warps_per_query=0) -> N.SearchParams:
        """Search parameters. ``L_query``, if given, must be a C-contiguous
        uint32 array kept alive by the caller until the call returns."""
        lq = None if L_query is None else L_query.ctypes.data
        return N.SearchParams(mode, distance, K, L, M, T, L_local, X, warps_per_block, storage, flags, lq,
                              blocks_per_sm, warps_per_query)

    def search(self, queries: np.ndarray | None = None, *, K=100, L=100, mode=N.MODE_NSG_SEQ,
               distance=N.DIST_NORM_IP, M=1, T=1, L_local=0, X=1, init_ids=None,
               q_begin=0, nq=None, warps_per_block=0, storage=N.STORE_FP32, flags=0, L_query=None,
               blocks_per_sm=0, warps_per_query=0, out=None):
        """Search a batch. ``out`` (optional): a C-contiguous nq x K uint32
        array to write the ids into (e.g. a view of pinned host memory). With ``queries`` None the loaded queries
        [q_begin, q_begin + nq) are used. ``L_query``: optional per-query
        queue lengths (K <= L_query[i] <= L). Returns (ids [nq x K], stats dict)."""
        if L_query is not None:
            L_query = np.ascontiguousarray(L_query, dtype=np.uint32)
        p = self.params(mode, distance, K, L, M, T, L_local, X, warps_per_block, storage, flags, L_query,
                        blocks_per_sm, warps_per_query)
        st = N.Stats()
        ii = None
        if init_ids is not None:
            ii = np.ascontiguousarray(init_ids, dtype=np.uint32)
        if queries is None:
            nq = self.nq - q_begin if nq is None else nq
            out = np.empty((nq, K), dtype=np.uint32) if out is None else out
            N.check(self._lib.panns_search(self._h, ctypes.byref(p), N.ptr(ii) if ii is not None else None,
                                           q_begin, nq, N.ptr(out), ctypes.byref(st)))
        else:
            queries = np.ascontiguousarray(queries, dtype=np.float32)
            nq = queries.shape[0]
            out = np.empty((nq, K), dtype=np.uint32) if out is None else out
            N.check(self._lib.panns_search_host(self._h, ctypes.byref(p), N.ptr(queries), nq,
                                                N.ptr(ii) if ii is not None else None, N.ptr(out),
                                                ctypes.byref(st)))
        return out, st.as_dict()

    def search_device(self, queries, out, *, K=100, L=100, mode=N.MODE_NSG_SEQ,
                      distance=N.DIST_NORM_IP, M=1, T=1, L_local=0, X=1, init_ids=None,
                      warps_per_block=0, storage=N.STORE_FP32, flags=0, L_query=None, stream=None,
                      blocks_per_sm=0, warps_per_query=0):
        """Asynchronous search of device queries (a torch float32 CUDA tensor,
        nq x d) into ``out`` (a torch int32/uint32 CUDA tensor, nq x K, original
        ids), enqueued on ``stream`` (a torch.cuda.Stream; None = the handle's
        own stream)."""
        if L_query is not None:
            L_query = np.ascontiguousarray(L_query, dtype=np.uint32)
        p = self.params(mode, distance, K, L, M, T, L_local, X, warps_per_block, storage, flags, L_query,
                        blocks_per_sm, warps_per_query)
        ii = None if init_ids is None else np.ascontiguousarray(init_ids, dtype=np.uint32)
        s = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
        N.check(self._lib.panns_search_device(self._h, ctypes.byref(p), ctypes.c_void_p(queries.data_ptr()),
                                              queries.shape[0], N.ptr(ii) if ii is not None else None,
                                              ctypes.c_void_p(out.data_ptr()), s, None))


def ground_truth(index: "Index", queries: np.ndarray, k: int = 100):
    """Top-k original ids and float64 distances by exact brute force on the GPU."""
    queries = np.ascontiguousarray(queries, dtype=np.float32)
    nq = queries.shape[0]
    ids = np.empty((nq, k), dtype=np.uint32)
    dist = np.empty((nq, k), dtype=np.float64)
    N.check(index._lib.panns_ground_truth(index._h, N.ptr(queries), nq, k, N.ptr(ids), N.ptr(dist)))
    return ids, dist


def recall(result_ids: np.ndarray, true_ids: np.ndarray, L: int, at: int = 100) -> float:
    r = np.ascontiguousarray(result_ids, dtype=np.uint32)
    t = np.ascontiguousarray(true_ids, dtype=np.uint32)
    out = ctypes.c_double()
    N.check(N.load().panns_recall(N.ptr(r), r.shape[0], r.shape[1], N.ptr(t), t.shape[1], L, at,
                                  ctypes.byref(out)))
    return out.value


class Searching:
    """``PANNS::Searching`` with the reference's method names.

    ``load_nsg_graph`` selects the norm-trick distance of the small-graph
    engine; ``load_common_nsg_graph`` the full L2 of the large-graph engine.
    Per-query methods keep the reference signatures (scratch arguments such as
    ``set_L``, ``local_queues_*`` and ``is_visited`` are accepted and ignored:
    that state lives on the GPU); each call is one GPU launch, so the
    ``*_batch`` forms are the fast path.
    """

    def __init__(self, device: int = 0):
        self.index = Index(device)
        self.num_v_ = 0
        self.num_queries_ = 0
        self.dimension_ = 0
        self.width_ = 0
        self.ep_ = 0
        self.num_threads_ = 1
        self.index_thresh_ = 99
        self.count_distance_computation_ = 0
        self.count_merge_ = 0
        self.time_expand_ = 0.0
        self.time_merge_ = 0.0
        self.time_seq_ = 0.0
        self._distance = N.DIST_NORM_IP
        self.last_stats = {}

    def _sync(self):
        i = self.index.info()
        self.num_v_, self.dimension_, self.num_queries_ = i["n"], i["d"], i["nq"]
        self.width_, self.ep_ = i["width"], i["entry"]

    def load_data_load(self, filename: str):
        self.index.load_fvecs_base(filename)
        self._sync()

    def load_queries_load(self, filename: str):
        self.index.load_fvecs_queries(filename)
        self._sync()

    def load_nsg_graph(self, filename: str):
        self.index.load_nsg(filename)
        self._distance = N.DIST_NORM_IP
        self._sync()

    def load_common_nsg_graph(self, filename: str):
        self.index.load_nsg(filename)
        self._distance = N.DIST_L2
        self._sync()

    def prepare_init_ids(self, init_ids: list, L: int):
        ids = self.index.prepare_init_ids(L)
        init_ids[:] = [int(x) for x in ids]

    def load_true_NN(self, filename: str, true_nn_list: list):
        ids, _ = read_true_nn(filename)
        if ids.shape[0] < self.num_queries_:
            raise N.PannsError(-2, f"t_query_num {ids.shape[0]} is smaller than num_queries_ "
                                   f"{self.num_queries_}")
        if ids.shape[1] < 100:
            raise N.PannsError(-2, f"t_K {ids.shape[1]} is smaller than 100.")
        true_nn_list[:] = [list(r) for r in ids]

    def get_recall_for_all_queries(self, true_nn_list, set_K_list, recalls: dict, L: int):
        t = np.asarray(true_nn_list, dtype=np.uint32)[: self.num_queries_]
        r = np.asarray(set_K_list, dtype=np.uint32)[: self.num_queries_]
        if t.shape[1] < 100:
            raise N.PannsError(-1, "Number of true nearest neighbors of a query is smaller than 100.")
        for at in (1, 5, 10, 20, 50, 100):
            recalls[at] = recall(r, t, L, at) if r.shape[1] >= 1 else 0.0

    # -- batched forms ------------------------------------------------------
    def _run(self, mode, K, L, init_ids=None, q_begin=0, nq=None, **kw):
        ids, st = self.index.search(None, K=K, L=L, mode=mode, distance=self._distance,
                                    init_ids=init_ids, q_begin=q_begin, nq=nq, **kw)
        self.count_distance_computation_ += st["n_dist"]
        self.last_stats = st
        return ids

    def para_search_PSS_v5_batch(self, K, L, init_ids, L_local, X, q_begin=0, nq=None):
        return self._run(N.MODE_PSS_V5, K, L, init_ids, q_begin, nq, T=self.num_threads_,
                         L_local=L_local, X=X)

    def seq_search_simple_search_batch(self, K, L, init_ids, q_begin=0, nq=None):
        return self._run(N.MODE_NSG_SEQ, K, L, init_ids, q_begin, nq)

    def para_search_with_top_m_pure_batch(self, M, K, L, init_ids, q_begin=0, nq=None):
        return self._run(N.MODE_TOP_M, K, L, init_ids, q_begin, nq, M=M)

    # -- per-query forms, reference signatures --------------------------------
    def para_search_PSS_v5_dist_thresh_profiling(self, query_id, K, L, set_L, init_ids, set_K,
                                                 local_queue_capacity, local_queues_starts,
                                                 local_queues_sizes, is_visited,
                                                 subsearch_iterations):
        ids = self.para_search_PSS_v5_batch(K, L, init_ids, local_queue_capacity,
                                            subsearch_iterations, query_id, 1)
        set_K[:K] = [int(x) for x in ids[0]]

    para_search_PSS_v5_large_graph_dist_thresh_profiling = para_search_PSS_v5_dist_thresh_profiling

    def seq_search_simple_search(self, query_id, K, L, set_L, init_ids, set_K, is_visited):
        ids = self.seq_search_simple_search_batch(K, L, init_ids, query_id, 1)
        set_K[:K] = [int(x) for x in ids[0]]

    def para_search_with_top_m_pure(self, M, query_id, K, L, set_L, init_ids, set_K,
                                    local_queue_capacity, local_queues_starts, local_queues_sizes,
                                    top_m_candidates, is_visited):
        ids = self.para_search_with_top_m_pure_batch(M, K, L, init_ids, query_id, 1)
        set_K[:K] = [int(x) for x in ids[0]]

    def seq_search_with_top_m_pure(self, M, query_id, K, L, set_L, init_ids, set_K,
                                   top_m_candidates, is_visited):
        ids = self.para_search_with_top_m_pure_batch(M, K, L, init_ids, query_id, 1)
        set_K[:K] = [int(x) for x in ids[0]]


class IndexNSG:
    """efanna2e::IndexNSG query path (include/efanna2e/index_nsg.h:17-43)."""

    def __init__(self, dimension: int, n: int, metric: int = 0, initializer=None, device: int = 0):
        self.dimension_ = dimension
        self.nd_ = n
        self.index = Index(device)
        self.count_distance_computation_ = 0
        self.count_iters_ = 0
        self._rand = Index.rand_state(1)  # the never-seeded process rand()
        self._base_set = False
        self._opt = False

    def Load(self, filename: str):
        self.index.load_nsg(filename)

    def OptimizeGraph(self, data: np.ndarray):
        self.index.set_base(np.asarray(data, dtype=np.float32).reshape(self.nd_, self.dimension_))
        self._base_set = True
        self._opt = True

    def _search(self, queries, K, L, distance):
        queries = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, self.dimension_)
        init = self.index.efanna_init_ids(L, queries.shape[0], self._rand)
        ids, st = self.index.search(queries, K=K, L=L, mode=N.MODE_EFANNA, distance=distance,
                                    init_ids=init)
        self.count_distance_computation_ += st["n_dist"]
        self.count_iters_ += st["n_expand"]
        return ids

    def Search(self, query, x, K, L_search, indices=None):
        """IndexNSG::Search (full L2 on the raw data x)."""
        if not self._base_set:
            self.index.set_base(np.asarray(x, dtype=np.float32).reshape(self.nd_, self.dimension_))
            self._base_set = True
        ids = self._search(query, K, L_search, N.DIST_L2)
        if indices is not None:
            indices[:K] = ids[0]
        return ids

    def SearchWithOptGraph(self, query, K, L_search, indices=None):
        """IndexNSG::SearchWithOptGraph (norm-trick distance)."""
        if not self._opt:
            raise N.PannsError(-5, "OptimizeGraph must be called first")
        ids = self._search(query, K, L_search, N.DIST_NORM_IP)
        if indices is not None:
            indices[:K] = ids[0]
        return ids

    def SearchBatch(self, queries, K, L_search, opt=True):
        """All queries in one launch; the rand() stream advances as if the
        queries had been searched one by one in order."""
        return self._search(queries, K, L_search, N.DIST_NORM_IP if opt else N.DIST_L2)
