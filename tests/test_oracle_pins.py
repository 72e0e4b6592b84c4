"""The CPU oracle is pinned to the reference: it must reproduce, bit for bit,
the reference's distances and norms and, id for id, the result lists and
distance counts the reference produced for the committed golden fixtures
(tests/golden/, generated by tests/golden/make_golden.py from the reference
sources). Where the reference binaries are present (oracle/_ref), they
are re-run and must reproduce the fixtures too."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, golden_ids, load_case

CASES = ["mix3k_d96", "mix1k_d24", "u8_1k_d128"]


def _oracle_run(form, spec, base, q, G):
    a = spec["args"]
    b = spec["binary"]
    K, L = a["K"], a["L"]
    if b in ("ref_pss", "ref_pss_lg"):
        kind = O.DIST_IP_NORM if b == "ref_pss" else O.DIST_L2
        return O.search_pss(base, G, q, K, L, a.get("L_local", L), a["X"], a["T"], kind=kind)
    if b == "ref_topm":
        M = a.get("M", 1) if a["mode"] != "simple" else 1
        return O.search_top_m(base, G, q, K, L, M)
    kind = O.DIST_L2 if a["mode"] == "search" else O.DIST_IP_NORM
    return O.search_efanna(base, G, q, K, L, kind=kind)


@pytest.mark.parametrize("case", CASES)
def test_distance_bits_match_reference(case):
    base, q, g, _ = load_case(case)
    d = os.path.join(GOLDEN, case)
    ids = np.fromfile(os.path.join(d, "dist_ids.u32"), dtype=np.uint32)
    ref_norm = np.fromfile(os.path.join(d, "norms.f32"), dtype=np.float32)
    nrm = O.norms(base)
    assert np.array_equal(nrm[ids].view(np.uint32), ref_norm.view(np.uint32))
    for fname, kind in (("dist_ip.f32", O.DIST_IP_NORM), ("dist_l2.f32", O.DIST_L2)):
        ref = np.fromfile(os.path.join(d, fname), dtype=np.float32).reshape(-1, ids.size)
        got = np.array([[O.distance(base[i], q[j], nrm[i], kind) for i in ids]
                        for j in range(ref.shape[0])], dtype=np.float32)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), fname


def test_unfused_lane_steps_do_not_match():
    """The pin is meaningful: separate multiply and add give other bits."""
    base, q, g, _ = load_case("mix3k_d96")
    d = os.path.join(GOLDEN, "mix3k_d96")
    ids = np.fromfile(os.path.join(d, "dist_ids.u32"), dtype=np.uint32)
    ref = np.fromfile(os.path.join(d, "dist_l2.f32"), dtype=np.float32).reshape(-1, ids.size)
    got = np.array([[O.distance(base[i], q[j], 0.0, O.DIST_L2, fused=0) for i in ids]
                    for j in range(ref.shape[0])], dtype=np.float32)
    assert (got != ref).sum() > 0


@pytest.mark.parametrize("case", CASES)
def test_oracle_reproduces_reference_ids(case, golden_manifest):
    base, q, g, _ = load_case(case)
    G = O.Graph.from_nsg(g)
    for form, spec in golden_manifest[case]["forms"].items():
        got, nd = _oracle_run(form, spec, base, q, G)
        ref = golden_ids(case, form, spec["args"]["K"])
        assert np.array_equal(got, ref), f"{case}/{form}: {(got != ref).any(1).sum()} rows differ"
        assert nd == spec["n_dist"], f"{case}/{form}: n_dist {nd} != {spec['n_dist']}"


@pytest.mark.skipif(not O.have_ref(), reason="reference binaries not built here")
@pytest.mark.parametrize("case", ["mix3k_d96", "mix1k_d24"])
def test_reference_binaries_reproduce_fixtures(case, golden_manifest):
    d = os.path.join(GOLDEN, case)
    files = dict(data=os.path.join(d, "base.fvecs"), queries=os.path.join(d, "query.fvecs"),
                 nsg=os.path.join(d, "graph.nsg"))
    with tempfile.TemporaryDirectory() as tmp:
        for form, spec in golden_manifest[case]["forms"].items():
            ids, st = O.run_ref(spec["binary"], os.path.join(tmp, "o.ids"), **files, **spec["args"])
            assert np.array_equal(ids, golden_ids(case, form, spec["args"]["K"])), form
            assert st["n_dist"] == spec["n_dist"], form


def test_rand_replay_matches_libc():
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(1)
    r = O.Rand(1)
    assert all(libc.rand() == r() for _ in range(20000))
    libc.srand(12345)
    r = O.Rand(12345)
    assert all(libc.rand() == r() for _ in range(2000))


def test_prepare_init_ids_rules():
    # entry 2 with neighbours [5, 5, 1] and N = 8: dedup, then 3, 4, ... wrapping
    from parallel_anns_b200.formats import NSGGraph
    g = NSGGraph.from_lists(3, 2, [[1], [2], [5, 5, 1], [], [], [0], [], []])
    G = O.Graph.from_nsg(g)
    assert O.prepare_init_ids(G, 6).tolist() == [5, 1, 3, 4, 6, 7]
    assert O.prepare_init_ids(G, 8).tolist() == [5, 1, 3, 4, 6, 7, 0, 2]


def test_pss_many_workers_recall_close_to_single(golden_manifest):
    """PSS_v5 with several queues (deterministic round-robin schedule) stays
    within a hair of the one-queue recall, as the reference does at T > 1."""
    base, q, g, tid = load_case("mix3k_d96")
    G = O.Graph.from_nsg(g)
    r1, _ = O.search_pss(base, G, q, 100, 200, 200, 1, 1)
    base_rec = O.recall_at(r1, tid, 200)
    for T, X in ((2, 1), (4, 2), (8, 4)):
        rt, _ = O.search_pss(base, G, q, 100, 200, 200, X, T)
        assert abs(O.recall_at(rt, tid, 200) - base_rec) < 0.01


@pytest.mark.skipif(not O.have_ref(), reason="reference binaries not built here")
@pytest.mark.parametrize("T,X", [(2, 1), (4, 2), (8, 4)])
def test_pss_workers_against_reference(T, X):
    """PSS_v5 at T > 1 is not deterministic in the reference (its workers race
    on the shared visited bitset). The fixed round-robin schedule used by the
    oracle and the GPU must keep the reference's recall; per-query overlap of
    the id sets is reported."""
    base, q, g, tid = load_case("mix3k_d96")
    G = O.Graph.from_nsg(g)
    d = os.path.join(GOLDEN, "mix3k_d96")
    files = dict(data=os.path.join(d, "base.fvecs"), queries=os.path.join(d, "query.fvecs"),
                 nsg=os.path.join(d, "graph.nsg"))
    ours, _ = O.search_pss(base, G, q, 100, 200, 200, X, T)
    with tempfile.TemporaryDirectory() as tmp:
        ref, st = O.run_ref("ref_pss", os.path.join(tmp, "o.ids"), **files, K=100, L=200, T=T, X=X)
    r_ours, r_ref = O.recall_at(ours, tid, 200), O.recall_at(ref, tid, 200)
    overlap = np.mean([np.intersect1d(a, b).size / 100.0 for a, b in zip(ours, ref)])
    print(f"T={T} X={X}: recall ours {r_ours:.4f} ref {r_ref:.4f}, mean id overlap {overlap:.4f}")
    assert r_ours >= r_ref - 0.005
    assert overlap > 0.95


@pytest.mark.skipif(not os.path.exists(os.path.join(O.REF_DIR, "ref_multi")),
                    reason="reference inter-query binary not built here")
@pytest.mark.parametrize("T", [1, 4])
def test_reference_inter_query_mode_reproduces_fixtures(T, golden_manifest):
    """The reference's inter-query PSS_v5 (multi_queries_LG, one thread per
    query, T queries at a time) returns the LG engine's single-thread ids and
    distance counts: the CPU baseline runs the same search."""
    d = os.path.join(GOLDEN, "mix3k_d96")
    files = dict(data=os.path.join(d, "base.fvecs"), queries=os.path.join(d, "query.fvecs"),
                 nsg=os.path.join(d, "graph.nsg"))
    for form in ("lg_t1_L100", "lg_t1_L250"):
        spec = golden_manifest["mix3k_d96"]["forms"][form]
        a = spec["args"]
        with tempfile.TemporaryDirectory() as tmp:
            ids, st = O.run_ref("ref_multi", os.path.join(tmp, "o.ids"), **files, K=a["K"], L=a["L"], T=T,
                                X=a["X"], inner=1)
        assert np.array_equal(ids, golden_ids("mix3k_d96", form, a["K"])), form
        assert st["n_dist"] == spec["n_dist"], form
