"""The host-side builder of the benchmark's inputs (oracle/host_build.c),
which the reference arm of the benchmark uses so that its process never maps
the GPU library: the same graph as the brute-force construction po_build_nsg
(k-NN lists, adjacency, entry, width) and the same top-k as the brute-force
float64 ground truth, on mixtures large enough for several clusters."""
import numpy as np
import pytest

import oracle as O


@pytest.mark.parametrize("n,d,seed", [(6000, 96, 5), (5000, 24, 6), (3000, 128, 7)])
def test_host_build_equals_brute_force(n, d, seed):
    from parallel_anns_b200 import datasets as ds
    base = ds.gaussian_mixture(n, d, seed=seed, means_seed=seed)
    g, knn = O.build_nsg(base, 64, 50)
    h, hknn = O.host_build_nsg(base, 64, 50)
    assert (h.entry, h.width) == (g.entry, g.width)
    assert np.array_equal(h.offsets, g.offsets) and np.array_equal(h.nbrs, g.nbrs)
    assert np.array_equal(hknn, knn)


def test_host_knn_equals_brute_force_ground_truth():
    from parallel_anns_b200 import datasets as ds
    base = ds.gaussian_mixture(8000, 96, seed=9, means_seed=9)
    q = ds.gaussian_mixture(200, 96, seed=10, means_seed=9)
    ids, dist = O.ground_truth(base, q, 100)
    hids, hdist = O.host_knn(base, q, 100)
    assert np.array_equal(hids, ids)
    assert np.allclose(hdist, dist, rtol=1e-12, atol=1e-15)


def test_host_knn_with_duplicate_rows():
    """Exact ties (duplicated rows) are broken by id, as in the brute force."""
    rng = np.random.default_rng(3)
    base = rng.standard_normal((5000, 32)).astype(np.float32)
    base[2500:2600] = base[:100]
    g, knn = O.build_nsg(base, 32, 24)
    h, hknn = O.host_build_nsg(base, 32, 24)
    assert np.array_equal(hknn, knn) and np.array_equal(h.nbrs, g.nbrs) and h.entry == g.entry
