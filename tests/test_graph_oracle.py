"""The graph-construction oracle (po_build_nsg, plain C) against a direct numpy
restatement on small inputs: exact float64 k-NN by (distance, id), the MRNG
pruning rule, the medoid entry and the reachability repair."""
import numpy as np

import oracle as O


def numpy_build(x, k, R):
    from parallel_anns_b200.datasets import repair_reachability
    n = x.shape[0]
    x64 = x.astype(np.float64)
    D = ((x64[:, None, :] - x64[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(D, np.inf)
    knn = np.array([np.lexsort((np.arange(n), D[a]))[:k] for a in range(n)], dtype=np.uint32)
    lists = []
    for a in range(n):
        kept = []
        for b in knn[a]:
            if len(kept) == R:
                break
            if not any(D[c, b] < D[a, b] for c in kept):
                kept.append(int(b))
        lists.append(np.array(kept, dtype=np.uint32))
    mean = x64.sum(0) / n
    dm = ((x64 - mean) ** 2).sum(1)
    entry = int(np.lexsort((np.arange(n), dm))[0])
    repair_reachability(lists, entry, knn)
    return lists, entry, knn


def test_oracle_graph_matches_numpy_restatement():
    from parallel_anns_b200 import datasets as ds
    x = ds.gaussian_mixture(400, 16, n_components=8, seed=77, means_seed=77)
    g, knn = O.build_nsg(x, 24, 12)
    lists, entry, knn_np = numpy_build(x, 24, 12)
    assert np.array_equal(knn, knn_np)
    assert g.entry == entry
    for v in range(x.shape[0]):
        assert np.array_equal(g.neighbors(v), lists[v]), v
    assert g.width == max(len(l) for l in lists)


def test_oracle_graph_ties_by_id_and_repair():
    # duplicated rows: equal distances are ordered by id; a far cluster forces repairs
    rng = np.random.default_rng(5)
    a = rng.standard_normal((60, 8)).astype(np.float32)
    x = np.concatenate([a, a[:20], a[:5] + 50.0]).astype(np.float32)
    g, knn = O.build_nsg(x, 6, 3)
    lists, entry, knn_np = numpy_build(x, 6, 3)
    assert np.array_equal(knn, knn_np)
    assert g.entry == entry
    for v in range(x.shape[0]):
        assert np.array_equal(g.neighbors(v), lists[v]), v
