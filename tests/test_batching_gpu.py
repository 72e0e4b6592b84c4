"""Batching features of the search launch, through the C ABI: per-query queue
lengths (each query searches exactly as a call with that L would), the
asynchronous device-pointer entry point, and the CUDA-graph-captured launch
(replayed, updated on a new shape, identical ids). Ids are checked against the
CPU oracle and against the ordinary host entry point."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def N_lib():
    from parallel_anns_b200 import native as N
    return N


@pytest.fixture(scope="module")
def setup():
    from parallel_anns_b200 import datasets as ds
    from parallel_anns_b200 import native as N
    from parallel_anns_b200.searching import Index
    base = ds.gaussian_mixture(20000, 96, seed=401, means_seed=401)
    q = ds.gaussian_mixture(256, 96, seed=402, means_seed=401)
    g = ds.build_nsg_graph(base, R=50, knn_k=64, device="cpu")
    ix = Index(0)
    ix.set_base(base)
    ix.set_graph(g)
    ix.set_queries(q)
    yield ix, N, base, q, g
    ix.close()


@pytest.mark.parametrize("mode,M", [(0, 1), (1, 4)])
def test_per_query_L_equals_per_L_calls(setup, mode, M):
    ix, N, base, q, g = setup
    K, Lmax = 50, 300
    Lq = np.random.default_rng(7).choice([50, 64, 100, 171, 300], size=q.shape[0]).astype(np.uint32)
    got, st = ix.search(K=K, L=Lmax, mode=mode, M=M, L_query=Lq)
    n_dist = 0
    for L in np.unique(Lq):
        sel = np.nonzero(Lq == L)[0]
        ref, s = ix.search(q[sel], K=K, L=int(L), mode=mode, M=M)
        assert np.array_equal(got[sel], ref), f"L={L}"
        n_dist += s["n_dist"]
    assert st["n_dist"] == n_dist
    # and the oracle agrees for one group
    G = O.Graph.from_nsg(g)
    sel = np.nonzero(Lq == 171)[0][:20]
    ref, _ = O.search_top_m(base, G, q[sel], K, 171, M)
    assert np.array_equal(got[sel], ref)


def test_per_query_L_rejects_out_of_range(setup):
    ix, N, base, q, g = setup
    bad = np.full(q.shape[0], 40, np.uint32)  # below K
    with pytest.raises(N.PannsError) as e:
        ix.search(K=50, L=100, L_query=bad)
    assert e.value.code == -1
    bad[:] = 101  # above L
    with pytest.raises(N.PannsError):
        ix.search(K=50, L=100, L_query=bad)
    with pytest.raises(N.PannsError):
        ix.search(K=50, L=100, mode=N.MODE_PSS_V5, T=4, L_query=np.full(q.shape[0], 60, np.uint32))


def test_device_entry_point_and_graph_replay(setup):
    import torch
    ix, N, base, q, g = setup
    ref, _ = ix.search(q, K=100, L=200, mode=N.MODE_TOP_M, M=8)
    qd = torch.from_numpy(q).cuda()
    s = torch.cuda.Stream()
    for flags in (0, N.FLAG_CUDA_GRAPH, N.FLAG_CUDA_GRAPH):
        out = torch.full((q.shape[0], 100), -1, dtype=torch.int32, device="cuda")
        ix.search_device(qd, out, K=100, L=200, mode=N.MODE_TOP_M, M=8, flags=flags, stream=s)
        s.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)
    # a new shape (fewer queries, other L) updates the captured graph
    ref2, _ = ix.search(q[:37], K=10, L=64)
    out2 = torch.full((37, 10), -1, dtype=torch.int32, device="cuda")
    ix.search_device(qd[:37], out2, K=10, L=64, flags=N.FLAG_CUDA_GRAPH, stream=s)
    s.synchronize()
    assert np.array_equal(out2.cpu().numpy().view(np.uint32), ref2)
    # host entry point with the graph flag, repeated
    for _ in range(2):
        got, _ = ix.search(q, K=100, L=200, mode=N.MODE_TOP_M, M=8, flags=N.FLAG_CUDA_GRAPH)
        assert np.array_equal(got, ref)


def test_single_query_batches(setup):
    """Batch size 1 through the graph-replayed device path, query by query."""
    import torch
    ix, N, base, q, g = setup
    ref, _ = ix.search(q[:16], K=100, L=128)
    qd = torch.from_numpy(q[:16]).cuda()
    out = torch.full((16, 100), -1, dtype=torch.int32, device="cuda")
    for i in range(16):
        ix.search_device(qd[i:i + 1], out[i:i + 1], K=100, L=128, flags=N.FLAG_CUDA_GRAPH)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)


def test_warps_per_block_beyond_kernel_limit_rejected(setup):
    ix, N, base, q, g = setup
    with pytest.raises(N.PannsError) as e:
        ix.search(K=10, L=64, warps_per_block=8)
    assert e.value.code == -1
    a, _ = ix.search(K=10, L=64, warps_per_block=2)
    b, _ = ix.search(K=10, L=64, warps_per_block=1)
    assert np.array_equal(a, b)
    c, _ = ix.search(K=10, L=64, warps_per_block=4, blocks_per_sm=1)  # fewer resident blocks: same ids
    assert np.array_equal(a, c)


def test_autotuner_meets_target_on_tuning_queries(setup):
    from parallel_anns_b200 import autotune as AT
    from parallel_anns_b200.searching import ground_truth, recall
    ix, N, base, q, g = setup
    gt, _ = ground_truth(ix, q, 100)
    c = AT.tune(ix, q, gt, K=100, target=0.97, Ms=(1, 4), wpbs=(2, 4), bpss=(0, 4), reps=1)
    assert c.recall >= 0.97 and c.M in (1, 4) and c.warps_per_block in (2, 4)
    ids, _ = ix.search(q, K=100, **c.search_kwargs())
    assert recall(ids, gt, 100, 100) == pytest.approx(c.recall)
    # every timed row reached the target; the choice is the fastest of them
    rows = [r for r in c.table if r.get("L")]
    assert all(r["recall"] >= 0.97 for r in rows)
    assert c.kernel_ms == min(r["kernel_ms"] for r in rows)


@pytest.mark.parametrize("wpq", [2, 4, 8])
@pytest.mark.parametrize("mode,M,L,dist", [(0, 1, 100, 0), (1, 4, 200, 0), (1, 8, 300, 1), (1, 64, 160, 0),
                                          (2, 1, 257, 1)])
def test_several_warps_per_query_equal_one(setup, wpq, mode, M, L, dist):
    """warps_per_query 2 / 4 return the one-warp kernel's ids and counts (and the oracle's)."""
    ix, N, base, q, g = setup
    K = min(100, L)
    ref, st = ix.search(K=K, L=L, mode=mode, M=M, distance=dist, warps_per_query=1)
    got, st2 = ix.search(K=K, L=L, mode=mode, M=M, distance=dist, warps_per_query=wpq)
    assert np.array_equal(got, ref)
    assert st2["n_dist"] == st["n_dist"] and st2["n_iter"] == st["n_iter"]
    assert st2["n_edges"] == st["n_edges"] and st2["n_expand"] == st["n_expand"]
    if mode == 1 and M == 8:
        G = O.Graph.from_nsg(g)
        oref, nd = O.search_top_m(base, G, q[:40], K, L, M, kind=O.DIST_L2)
        assert np.array_equal(got[:40], oref)


def test_several_warps_per_query_small_batches_and_per_query_L(setup):
    import torch
    ix, N, base, q, g = setup
    Lq = np.random.default_rng(3).choice([64, 100, 200], size=q.shape[0]).astype(np.uint32)
    ref, _ = ix.search(K=50, L=200, mode=1, M=8, L_query=Lq, warps_per_query=1)
    got, _ = ix.search(K=50, L=200, mode=1, M=8, L_query=Lq, warps_per_query=4)
    assert np.array_equal(got, ref)
    qd = torch.from_numpy(q[:5]).cuda()
    out = torch.full((5, 50), -1, dtype=torch.int32, device="cuda")
    for i in range(5):
        ix.search_device(qd[i:i + 1], out[i:i + 1], K=50, L=200, mode=1, M=8, warps_per_query=4,
                         flags=N.FLAG_CUDA_GRAPH)
    torch.cuda.synchronize()
    ref5, _ = ix.search(q[:5], K=50, L=200, mode=1, M=8)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref5)
    with pytest.raises(N.PannsError):
        ix.search(K=50, L=200, warps_per_query=3)
    with pytest.raises(N.PannsError):
        ix.search(K=50, L=200, mode=N.MODE_EFANNA, warps_per_query=2)
    with pytest.raises(N.PannsError):
        ix.search(K=50, L=200, mode=N.MODE_TOP_M, M=4, warps_per_query=2, flags=N.FLAG_LEARNED)


@pytest.mark.parametrize("d", [8, 24, 128, 256])
def test_several_warps_per_query_dimensions(N_lib, d):
    from parallel_anns_b200 import datasets as ds
    from parallel_anns_b200.searching import Index
    base = ds.gaussian_mixture(3000, d, seed=d, means_seed=d)
    q = ds.gaussian_mixture(64, d, seed=d + 1, means_seed=d)
    g = ds.build_nsg_graph(base, R=32, knn_k=40, device="cpu")
    with Index(0) as ix:
        ix.set_base(base)
        ix.set_graph(g)
        ix.set_queries(q)
        for dist in (0, 1):
            ref, st = ix.search(K=50, L=120, mode=1, M=4, distance=dist, warps_per_query=1)
            got, st2 = ix.search(K=50, L=120, mode=1, M=4, distance=dist, warps_per_query=2)
            assert np.array_equal(got, ref) and st["n_dist"] == st2["n_dist"]


def test_long_queue_default_block_shape(setup):
    """L = 8192: four one-warp queues do not fit a block's shared memory, so the
    default block shape shrinks (an explicit 4 is rejected); ids equal the oracle's."""
    ix, N, base, q, g = setup
    with pytest.raises(N.PannsError):
        ix.search(q[:8], K=100, L=8192, mode=N.MODE_TOP_M, M=8, warps_per_block=4)
    got, _ = ix.search(q[:8], K=100, L=8192, mode=N.MODE_TOP_M, M=8)
    ref, _ = O.search_top_m(base, O.Graph.from_nsg(g), q[:8], 100, 8192, 8)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("storage", [1, 2])
def test_several_warps_per_query_reduced_storage(storage):
    """BF16 / FP8 copies with 2 and 4 warps per query: same ids and counts as
    one warp per query on the same copy (same distances, same re-rank)."""
    from parallel_anns_b200 import datasets as ds
    from parallel_anns_b200 import native as N
    from parallel_anns_b200.searching import Index
    base = ds.gaussian_mixture(20000, 96, seed=411, means_seed=411)
    q = ds.gaussian_mixture(200, 96, seed=412, means_seed=411)
    g = ds.build_nsg_graph(base, R=50, knn_k=64, device="cpu")
    with Index(0) as ix:
        ix.set_base(base, storage=storage)
        ix.set_graph(g)
        ix.set_queries(q)
        for L, M, K in ((200, 8, 100), (257, 4, 10)):
            ref, st = ix.search(K=K, L=L, mode=N.MODE_TOP_M, M=M, storage=storage, warps_per_query=1)
            for wq in (2, 4, 8):
                got, st2 = ix.search(K=K, L=L, mode=N.MODE_TOP_M, M=M, storage=storage, warps_per_query=wq)
                assert np.array_equal(got, ref), (storage, L, wq)
                assert st2["n_dist"] == st["n_dist"]
