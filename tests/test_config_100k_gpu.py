"""Id parity at the small benchmark configuration, against the reference's own
binaries run here (oracle/_ref/ref_*, built from the reference sources).

Workload: N = 100,000 vectors, d = 96, 64-component Gaussian mixture (sigma
0.3, unit norm), 1,000 queries from the same mixture, NSG-style graph R = 50
(exact 64-NN, MRNG prune, medoid entry, reachability repair), K = 100,
L in {100, 200, 400}. Forms, each with the reference's distance:
  * sequential NSG search, core/Searching.202011241533.top_m_pure.cpp:1486-1605
    (seq_search_simple_search) — NSG_SEQ, norm-trick distance;
  * PSS_v5 at one thread,
    core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp:1218-1515, and
    its large-graph twin (full L2),
    core/Searching.202102031939.PSS_v5.large_graph.dist_thresh.profiling.cpp:1376-1726;
  * top-M search with M = 64 at one thread, top_m_pure.cpp:1881-2070;
  * efanna2e IndexNSG::Search (L2) and SearchWithOptGraph (norm trick) with
    the rand() initial ids, include/efanna2e/index_nsg.cpp:452-611.
Every id of every row and the total distance count must equal the
reference's. A mismatch would be tolerated only between two distances that
tie within 1e-6 relative; none is expected (the GPU computes the same float32
bits), and any is reported with its distances.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

LS = (100, 200, 400)


@pytest.fixture(scope="module")
def workload(tmp_path_factory):
    if not O.have_ref():
        pytest.skip("reference binaries not built (oracle/_ref)")
    from parallel_anns_b200 import formats as fm
    from parallel_anns_b200 import workloads
    from parallel_anns_b200.graph import build_nsg
    spec = workloads.SPECS["mixture_1m_d96"](n=100_000, nq=1_000)
    base = workloads.vectors(spec, spec["n"], spec["base_seed"])
    q = workloads.vectors(spec, spec["nq"], spec["query_seed"])
    g = build_nsg(base, R=spec["R"], knn_k=spec["knn_k"], device=0)
    h, _ = O.host_build_nsg(base, spec["knn_k"], spec["R"])
    assert (g.entry, g.width) == (h.entry, h.width)
    assert np.array_equal(g.offsets, h.offsets) and np.array_equal(g.nbrs, h.nbrs)
    d = tmp_path_factory.mktemp("cfg100k")
    paths = {"data": str(d / "base.fvecs"), "queries": str(d / "query.fvecs"), "nsg": str(d / "graph.nsg")}
    fm.write_fvecs(paths["data"], base)
    fm.write_fvecs(paths["queries"], q)
    fm.write_nsg(paths["nsg"], g)
    return base, q, g, paths, d


@pytest.fixture(scope="module")
def index(workload):
    from parallel_anns_b200.searching import Index
    base, q, g, _, _ = workload
    ix = Index(0)
    ix.set_base(base)
    ix.set_graph(g)
    ix.set_queries(q)
    yield ix
    ix.close()


def ties_only(base, q, ids, ref, name):
    """True if every differing position holds two vertices whose distances
    tie within 1e-6 relative (each one printed)."""
    ok = True
    for r in np.nonzero((ids != ref).any(1))[0]:
        dq = lambda v: float(((base[v].astype(np.float64) - q[r]) ** 2).sum())
        for x, y in zip(ids[r], ref[r]):
            if x != y:
                dx, dy = dq(int(x)), dq(int(y))
                tie = abs(dx - dy) <= 1e-6 * max(dx, dy)
                print(f"{name} row {r}: gpu {x} ({dx:.9g}) vs reference {y} ({dy:.9g}) tie={tie}")
                ok &= tie
    return ok


def check(ix_ids, st, ref_ids, ref_st, base, q, name):
    bad = np.nonzero((ix_ids != ref_ids).any(1))[0]
    if bad.size:
        assert ties_only(base, q, ix_ids, ref_ids, name), f"{name}: rows {bad[:8].tolist()} differ"
    assert int(st["n_dist"]) == int(ref_st["n_dist"]), f"{name}: n_dist {st['n_dist']} vs {ref_st['n_dist']}"


@pytest.mark.parametrize("L", LS)
def test_sequential_and_pss_v5_t1(workload, index, L):
    from parallel_anns_b200 import native as N
    base, q, g, paths, d = workload
    out = str(d / f"seq_{L}.ids")
    ref, rst = O.run_ref("ref_topm", out, K=100, L=L, mode="simple", **paths)
    ids, st = index.search(K=100, L=L, mode=N.MODE_NSG_SEQ, distance=N.DIST_NORM_IP)
    check(ids, st, ref, rst, base, q, f"NSG_SEQ L={L}")
    ref, rst = O.run_ref("ref_pss", str(d / f"pss_{L}.ids"), K=100, L=L, T=1, X=1, **paths)
    ids, st = index.search(K=100, L=L, mode=N.MODE_PSS_V5, distance=N.DIST_NORM_IP, T=1, X=1)
    check(ids, st, ref, rst, base, q, f"PSS_v5 T=1 L={L}")
    ref, rst = O.run_ref("ref_pss_lg", str(d / f"lg_{L}.ids"), K=100, L=L, T=1, X=1, **paths)
    ids, st = index.search(K=100, L=L, mode=N.MODE_PSS_V5, distance=N.DIST_L2, T=1, X=1)
    check(ids, st, ref, rst, base, q, f"PSS_v5 LG T=1 L={L}")


@pytest.mark.parametrize("L", LS)
def test_top_m_64(workload, index, L):
    from parallel_anns_b200 import native as N
    base, q, g, paths, d = workload
    ref, rst = O.run_ref("ref_topm", str(d / f"topm_{L}.ids"), K=100, L=L, M=64, mode="topm_para", T=1,
                         **paths)
    for wpq in (1, 0):
        ids, st = index.search(K=100, L=L, mode=N.MODE_TOP_M, distance=N.DIST_NORM_IP, M=64, warps_per_query=wpq)
        check(ids, st, ref, rst, base, q, f"TOP_M M=64 L={L} wpq={wpq}")


@pytest.mark.parametrize("L", LS)
def test_efanna_search_and_opt(workload, index, L):
    from parallel_anns_b200 import native as N
    base, q, g, paths, d = workload
    for mode, dist in (("search", N.DIST_L2), ("opt", N.DIST_NORM_IP)):
        ref, rst = O.run_ref("ref_efanna", str(d / f"efanna_{mode}_{L}.ids"), K=100, L=L, mode=mode, **paths)
        ids, st = index.search(K=100, L=L, mode=N.MODE_EFANNA, distance=dist)
        check(ids, st, ref, rst, base, q, f"efanna {mode} L={L}")
