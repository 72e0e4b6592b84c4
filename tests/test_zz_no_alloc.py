"""panns_search_static: the search for callers that cannot allocate GPU memory
while running (e.g. a server whose device memory is all reserved by a
framework's pool, or a plug-in in a host that forbids allocations after
start-up). Its scratch lives in one fixed array of the library, so this test
checks, through the C ABI, that it returns exactly the ids of the ordinary
entry point on two calls in a row (the array keeps the previous call's
contents), and that sizes beyond its fixed limits are rejected.

Collected last on purpose (file name), so a run that stops at the first
failure has run every other test before this one."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    import torch
    from parallel_anns_b200 import datasets as ds
    from parallel_anns_b200.searching import Index
    base = ds.gaussian_mixture(20000, 96, seed=301, means_seed=301)
    q = ds.gaussian_mixture(500, 96, seed=302, means_seed=301)
    g = ds.build_nsg_graph(base, R=50, knn_k=64, device="cpu")
    ix = Index(0)
    ix.set_base(base)
    ix.set_graph(g)
    ix.set_queries(q)
    yield ix, q, torch
    ix.close()


def call_static(ix, torch, q_dev, out_dev, **kw):
    from parallel_anns_b200 import native as N
    p = ix.params(**kw)
    rc = N.load().panns_search_static(ix._h, ctypes.byref(p), ctypes.c_void_p(q_dev.data_ptr()),
                                      q_dev.shape[0], ctypes.c_void_p(out_dev.data_ptr()), None)
    return rc


@pytest.mark.parametrize("kw", [
    dict(mode=0, distance=0, K=100, L=160),
    dict(mode=1, distance=1, K=50, L=128, M=8),
])
def test_static_matches_ordinary_search_twice(setup, kw):
    from parallel_anns_b200 import native as N
    ix, q, torch = setup
    ref, _ = ix.search(**kw)  # ordinary entry point (also lays the index out on the GPU)
    q_dev = torch.from_numpy(q).cuda()
    for _ in range(2):
        out = torch.full((q.shape[0], kw["K"]), 0xFFFFFFFF, dtype=torch.int64).to(torch.int32).cuda()
        N.check(call_static(ix, torch, q_dev, out, **kw))
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, ref)


def test_static_rejects_sizes_beyond_its_limits(setup):
    from parallel_anns_b200 import native as N
    ix, q, torch = setup
    ix.search(K=10, L=20, nq=1)
    q_dev = torch.from_numpy(q).cuda()
    out = torch.zeros((q.shape[0], 100), dtype=torch.int32).cuda()
    rc = call_static(ix, torch, q_dev, out, K=100, L=2048)
    assert rc == -1 and b"fixed scratch" in N.load().panns_last_error()
    big = torch.zeros((120000, 96), dtype=torch.float32).cuda()
    out_big = torch.zeros((120000, 10), dtype=torch.int32).cuda()
    rc = call_static(ix, torch, big, out_big, K=10, L=20)
    assert rc == -1 and b"does not fit" in N.load().panns_last_error()


def test_static_overflowing_cleared_word_list_twice():
    """A query that sets more bitset words than the static path's cleared-word
    list holds (2048) falls back to clearing its whole bitset; the next call
    must still start from an empty visited set. A random graph of degree 128
    over N = 100,000 makes every query visit more than 65,536 vertices (its
    distance count), so more than 65,536 / 32 = 2048 words: the fallback runs
    on every query. Checked against the ordinary entry point and the CPU
    oracle, on two calls in a row."""
    import torch
    import oracle as O
    from parallel_anns_b200 import native as N
    from parallel_anns_b200.formats import NSGGraph
    from parallel_anns_b200.searching import Index
    rng = np.random.default_rng(404)
    n, d, deg, nq = 100_000, 16, 128, 24
    base = rng.standard_normal((n, d), dtype=np.float32)
    q = rng.standard_normal((nq, d), dtype=np.float32)
    lists = [rng.choice(n, size=deg, replace=False).astype(np.uint32) for _ in range(n)]
    g = NSGGraph.from_lists(deg, 0, lists)
    kw = dict(mode=0, distance=0, K=100, L=1024)
    with Index(0) as ix:
        ix.set_base(base)
        ix.set_graph(g)
        ix.set_queries(q)
        ref, st = ix.search(**kw)
        per_q = [ix.search(q_begin=i, nq=1, **kw)[1]["n_dist"] for i in range(nq)]
        assert min(per_q) > 65536, per_q
        oref, ond = O.search_top_m(base, O.Graph.from_nsg(g), q, 100, 1024, 1)
        assert np.array_equal(ref, oref) and st["n_dist"] == ond
        q_dev = torch.from_numpy(q).cuda()
        for _ in range(2):
            out = torch.zeros((nq, 100), dtype=torch.int32).cuda()
            N.check(call_static(ix, torch, q_dev, out, **kw))
            torch.cuda.synchronize()
            assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)


def test_static_rejects_launch_shapes_it_does_not_run(setup):
    from parallel_anns_b200 import native as N
    ix, q, torch = setup
    ix.search(K=10, L=20, nq=1)
    q_dev = torch.from_numpy(q).cuda()
    out = torch.zeros((q.shape[0], 100), dtype=torch.int32).cuda()
    for bad in (dict(warps_per_query=4), dict(blocks_per_sm=2)):
        rc = call_static(ix, torch, q_dev, out, K=100, L=128, **bad)
        assert rc == -1 and b"one warp per query" in N.load().panns_last_error()
