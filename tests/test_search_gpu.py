"""GPU parity of the search kernel, through the C ABI.

The bar is bit-exact: the GPU returns exactly the reference's id lists and
distance-computation counts. Checked against (1) the committed golden fixtures
produced by the reference itself and (2) the CPU oracle on freshly generated
seeded inputs, plus edge cases and error behaviour."""
import numpy as np
import pytest

import oracle as O
from conftest import golden_ids, load_case

pytestmark = pytest.mark.gpu

CASES = ["mix3k_d96", "mix1k_d24", "u8_1k_d128"]


@pytest.fixture(scope="module")
def N():
    from parallel_anns_b200 import native
    return native


def gpu_index(base, g, queries=None):
    from parallel_anns_b200.searching import Index
    ix = Index(0)
    ix.set_base(base)
    ix.set_graph(g)
    if queries is not None:
        ix.set_queries(queries)
    return ix


def gpu_form(ix, N, spec, wpq=0):
    """Run the GPU counterpart of a golden form (wpq: warps per query; 0 =
    the library's automatic choice, which for these small batches is a block
    of 8 warps per query where the form allows it)."""
    a, b = spec["args"], spec["binary"]
    K, L = a["K"], a["L"]
    if b in ("ref_pss", "ref_pss_lg"):
        dist = N.DIST_NORM_IP if b == "ref_pss" else N.DIST_L2
        return ix.search(K=K, L=L, mode=N.MODE_PSS_V5, distance=dist, T=a["T"], X=a["X"], warps_per_query=wpq)
    if b == "ref_topm":
        if a["mode"] == "simple":
            return ix.search(K=K, L=L, mode=N.MODE_NSG_SEQ, distance=N.DIST_NORM_IP, warps_per_query=wpq)
        return ix.search(K=K, L=L, mode=N.MODE_TOP_M, distance=N.DIST_NORM_IP, M=a["M"], warps_per_query=wpq)
    dist = N.DIST_L2 if a["mode"] == "search" else N.DIST_NORM_IP
    return ix.search(K=K, L=L, mode=N.MODE_EFANNA, distance=dist)


@pytest.mark.parametrize("wpq", [1, 0])
@pytest.mark.parametrize("case", CASES)
def test_gpu_matches_reference_golden(case, golden_manifest, N, wpq):
    base, q, g, _ = load_case(case)
    ix = gpu_index(base, g, q)
    for form, spec in golden_manifest[case]["forms"].items():
        ids, st = gpu_form(ix, N, spec, wpq)
        ref = golden_ids(case, form, spec["args"]["K"])
        bad = np.nonzero((ids != ref).any(1))[0]
        assert bad.size == 0, f"{case}/{form}: rows {bad[:8].tolist()} differ"
        assert st["n_dist"] == spec["n_dist"], f"{case}/{form}"
    ix.close()


@pytest.fixture(scope="module")
def mix20k():
    from parallel_anns_b200 import datasets as ds
    base = ds.gaussian_mixture(20000, 96, seed=101, means_seed=101)
    q = ds.gaussian_mixture(300, 96, seed=102, means_seed=101)
    g = ds.build_nsg_graph(base, R=50, knn_k=64, device="cpu")
    return base, q, g


@pytest.mark.parametrize("wpq", [1, 0])
@pytest.mark.parametrize("L,M", [(64, 1), (100, 1), (333, 1), (100, 2), (200, 8), (128, 32), (96, 64)])
def test_gpu_top_m_matches_oracle(mix20k, N, L, M, wpq):
    base, q, g = mix20k
    G = O.Graph.from_nsg(g)
    ix = gpu_index(base, g, q)
    K = min(100, L)
    mode = N.MODE_NSG_SEQ if M == 1 else N.MODE_TOP_M
    for dist, kind in ((N.DIST_NORM_IP, O.DIST_IP_NORM), (N.DIST_L2, O.DIST_L2)):
        ids, st = ix.search(K=K, L=L, mode=mode, distance=dist, M=M, warps_per_query=wpq)
        ref, nd = O.search_top_m(base, G, q, K, L, M, kind=kind)
        assert np.array_equal(ids, ref), f"L={L} M={M} dist={dist}: {(ids != ref).any(1).sum()} rows"
        assert st["n_dist"] == nd
    ix.close()


@pytest.mark.parametrize("L", [50, 150, 400])
def test_gpu_efanna_matches_oracle(mix20k, N, L):
    base, q, g = mix20k
    G = O.Graph.from_nsg(g)
    ix = gpu_index(base, g, q)
    init = ix.efanna_init_ids(L, q.shape[0])
    assert np.array_equal(init, O.efanna_init_ids(G, L, q.shape[0]))
    for dist, kind in ((N.DIST_L2, O.DIST_L2), (N.DIST_NORM_IP, O.DIST_IP_NORM)):
        ids, st = ix.search(K=50, L=L, mode=N.MODE_EFANNA, distance=dist, init_ids=init)
        ref, nd = O.search_efanna(base, G, q, 50, L, kind=kind, init_ids=init)
        assert np.array_equal(ids, ref)
        assert st["n_dist"] == nd
    ix.close()


def test_host_query_path_and_repeats(mix20k, N):
    """Queries passed as a host pointer give the same answers as loaded
    queries; repeated calls on one handle stay exact (visited sets are reset)."""
    base, q, g = mix20k
    ix = gpu_index(base, g, q)
    a, _ = ix.search(K=100, L=150)
    for _ in range(3):
        b, _ = ix.search(q, K=100, L=150)
        assert np.array_equal(a, b)
    c, _ = ix.search(K=100, L=150, q_begin=17, nq=40)
    assert np.array_equal(c, a[17:57])
    ix.close()


@pytest.mark.parametrize("d", [8, 24, 40, 128, 256])
def test_gpu_dimensions(N, d):
    from parallel_anns_b200 import datasets as ds
    base = ds.gaussian_mixture(1500, d, seed=d, means_seed=d)
    q = ds.gaussian_mixture(40, d, seed=d + 1, means_seed=d)
    g = ds.build_nsg_graph(base, R=24, knn_k=32, device="cpu")
    G = O.Graph.from_nsg(g)
    ix = gpu_index(base, g, q)
    for dist, kind in ((N.DIST_NORM_IP, O.DIST_IP_NORM), (N.DIST_L2, O.DIST_L2)):
        ids, st = ix.search(K=20, L=60, distance=dist)
        ref, nd = O.search_top_m(base, G, q, 20, 60, 1, kind=kind)
        assert np.array_equal(ids, ref)
        assert st["n_dist"] == nd
    ix.close()


@pytest.mark.parametrize("wpq", [1, 0])
def test_gpu_edge_graphs(N, wpq):
    """Zero-degree vertices, a hub with more neighbours than one head row holds,
    L = N (every vertex in the queue), K = 1, a single query."""
    from parallel_anns_b200.formats import NSGGraph
    rng = np.random.default_rng(5)
    n, d = 300, 32
    base = rng.standard_normal((n, d)).astype(np.float32)
    q = rng.standard_normal((7, d)).astype(np.float32)
    lists = [rng.choice(n, size=rng.integers(0, 6), replace=False).astype(np.uint32) for _ in range(n)]
    lists[0] = np.arange(1, 120, dtype=np.uint32)  # hub: 119 neighbours (head row + overflow)
    lists[5] = np.array([], dtype=np.uint32)
    g = NSGGraph.from_lists(119, 0, lists)
    G = O.Graph.from_nsg(g)
    ix = gpu_index(base, g, q)
    for L, K, M in ((10, 10, 1), (40, 1, 1), (n, 100, 1), (n, 5, 7), (64, 64, 64)):
        mode = N.MODE_NSG_SEQ if M == 1 else N.MODE_TOP_M
        for dist, kind in ((N.DIST_NORM_IP, O.DIST_IP_NORM), (N.DIST_L2, O.DIST_L2)):
            ids, st = ix.search(K=K, L=L, mode=mode, distance=dist, M=M, warps_per_query=wpq)
            ref, nd = O.search_top_m(base, G, q, K, L, M, kind=kind)
            assert np.array_equal(ids, ref), (L, K, M, dist)
            assert st["n_dist"] == nd
        one, _ = ix.search(q[3:4], K=K, L=L, mode=mode, M=M)
        ref1, _ = O.search_top_m(base, G, q[3:4], K, L, M)
        assert np.array_equal(one, ref1)
    ix.close()


def test_gpu_errors(mix20k, N):
    base, q, g = mix20k
    ix = gpu_index(base, g, q)
    with pytest.raises(N.PannsError, match="EINVAL"):
        ix.search(K=101, L=100)
    with pytest.raises(N.PannsError, match="EINVAL"):
        ix.search(K=10, L=base.shape[0] + 1)
    with pytest.raises(N.PannsError, match="EINVAL"):
        ix.search(K=10, L=20, init_ids=np.zeros(20, dtype=np.uint32))
    with pytest.raises(N.PannsError, match="EINVAL"):
        ix.search(K=10, L=20, init_ids=np.arange(20, dtype=np.uint32) + base.shape[0])
    with pytest.raises(N.PannsError, match="EINVAL"):
        ix.search(K=10, L=20, mode=N.MODE_TOP_M, M=0)
    with pytest.raises(N.PannsError, match="EINVAL"):
        ix.search(K=10, L=20, q_begin=290, nq=20)
    ids, st = ix.search(K=10, L=20, nq=0)
    assert ids.shape == (0, 10)
    # the handle still works after errors
    a, _ = ix.search(K=10, L=20, nq=5)
    ref, _ = O.search_top_m(base, O.Graph.from_nsg(g), q[:5], 10, 20, 1)
    assert np.array_equal(a, ref)
    ix.close()


@pytest.mark.parametrize("T,X,Ll", [(2, 1, 0), (4, 2, 0), (8, 4, 0), (3, 1, 64), (16, 8, 0), (5, 3, 300)])
def test_gpu_pss_workers_match_oracle(mix20k, N, T, X, Ll):
    """PSS_v5 with T queues: the GPU runs the oracle's fixed round-robin
    schedule, so ids and distance counts match exactly."""
    base, q, g = mix20k
    G = O.Graph.from_nsg(g)
    ix = gpu_index(base, g, q)
    L = 200
    for dist, kind in ((N.DIST_NORM_IP, O.DIST_IP_NORM), (N.DIST_L2, O.DIST_L2)):
        ids, st = ix.search(K=100, L=L, mode=N.MODE_PSS_V5, distance=dist, T=T, X=X, L_local=Ll)
        ref, nd = O.search_pss(base, G, q, 100, L, Ll or L, X, T, kind=kind)
        bad = np.nonzero((ids != ref).any(1))[0]
        assert bad.size == 0, f"T={T} X={X} Ll={Ll} dist={dist}: rows {bad[:8].tolist()}"
        assert st["n_dist"] == nd
    ix.close()


@pytest.mark.parametrize("storage", [1, 2])
def test_gpu_reduced_storage_recall_and_rerank(mix20k, N, storage):
    """BF16 / FP8-E4M3 storage: the search runs on the reduced copy, the final
    L are re-ranked with the exact FP32 distance. Recall@100 against the
    float64 ground truth must stay within 0.01 of the exact search at the same
    L, and the K results must be ordered by their exact distance, then id."""
    from parallel_anns_b200.searching import Index
    base, q, g = mix20k
    G = O.Graph.from_nsg(g)
    gt, _ = O.ground_truth(base, q, 100)
    ix = Index(0)
    ix.set_base(base, storage=storage)
    ix.set_graph(g)
    ix.set_queries(q)
    nrm = O.norms(base)
    # queue lengths cut into power-of-two runs by the re-rank: 128 | 128+64+8 | 256+1 | 64+32+4
    for L, M, K in ((128, 1, 100), (200, 4, 100), (257, 8, 100), (100, 2, 10)):
        mode = N.MODE_NSG_SEQ if M == 1 else N.MODE_TOP_M
        exact, _ = ix.search(K=K, L=L, mode=mode, M=M)
        red, st = ix.search(K=K, L=L, mode=mode, M=M, storage=storage)
        if K == 100:
            r_exact, r_red = O.recall_at(exact, gt, L), O.recall_at(red, gt, L)
            assert r_red >= r_exact - 0.01, (storage, L, M, r_red, r_exact)
        assert all(len(set(r.tolist())) == K for r in red)
        for row, qv in zip(red[:20], q[:20]):
            d = np.array([O.distance(base[i], qv, nrm[i], O.DIST_IP_NORM) for i in row], np.float32)
            key = list(zip(d.tolist(), row.tolist()))
            assert key == sorted(key)
    # exact float32 storage requested on a reduced handle still gives exact results
    ref, _ = O.search_top_m(base, G, q, 100, 128, 1)
    again, _ = ix.search(K=100, L=128)
    assert np.array_equal(again, ref)
    with pytest.raises(N.PannsError, match="EINVAL"):
        ix.search(K=100, L=128, storage=3 - storage)  # the other reduced copy was not built
    ix.close()


def test_gpu_fp64_ground_truth(mix20k):
    """The float64 brute-force kernel returns exactly the oracle's top-100
    (ties, if any, only where float64 distances agree to 1e-12 relative)."""
    from parallel_anns_b200.searching import Index, ground_truth
    base, q, g = mix20k
    ix = gpu_index(base, g)
    ids, dist = ground_truth(ix, q, 100)
    ref_ids, ref_d = O.ground_truth(base, q, 100)
    bad = np.nonzero((ids != ref_ids).any(1))[0]
    for r in bad:
        assert np.allclose(dist[r], ref_d[r], rtol=1e-12, atol=0), r
    assert np.allclose(dist, ref_d, rtol=1e-12, atol=0)
    assert bad.size <= 2
    ix.close()
