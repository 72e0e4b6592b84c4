"""The cell-restricted graph construction (panns_build_nsg_cells) on the GPU.

* With one cell it is the all-pairs construction: the graph equals
  panns_build_nsg with the float32 screen, byte for byte.
* With many cells every k-NN list equals a float64 brute force over the
  vertex's own cell and its probe nearest cells (the partition the build
  reports), up to the order of distances equal within 1e-9 relative.
* The pruned lists follow the MRNG rule on those k-NN lists, every vertex is
  reachable from the entry, and the entry is the vertex nearest the mean.
* With reverse edges every pruned edge a -> b is matched by b -> a unless b's
  list was full, and the lists still start with the pruned neighbours.
"""
from collections import deque

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _d2(a, B):
    a = a.astype(np.float64)
    B = B.astype(np.float64)
    t = B - a[None, :]
    return np.einsum("ij,ij->i", t, t)


def test_one_cell_equals_all_pairs_build():
    from parallel_anns_b200 import datasets as ds
    from parallel_anns_b200.graph import SCREEN_FP32, build_nsg, build_nsg_cells
    base = ds.gaussian_mixture(3000, 96, seed=61, means_seed=61)
    g1, k1 = build_nsg(base, R=24, knn_k=32, screen=SCREEN_FP32, with_knn=True)
    g2, k2 = build_nsg_cells(base, R=24, knn_k=32, cells=1, probe=0, sample=3000, iters=2, with_knn=True)
    assert np.array_equal(k1, k2)
    assert g1.entry == g2.entry and g1.width == g2.width
    assert np.array_equal(g1.offsets, g2.offsets) and np.array_equal(g1.nbrs, g2.nbrs)


@pytest.mark.parametrize("n,d,cells,probe,k,R", [(20000, 96, 32, 3, 32, 24), (6000, 24, 12, 2, 16, 12)])
def test_cell_knn_lists_prune_and_repair(n, d, cells, probe, k, R):
    from parallel_anns_b200 import datasets as ds
    from parallel_anns_b200.graph import build_nsg_cells
    base = ds.gaussian_mixture(n, d, seed=62 + d, means_seed=62 + d)
    g, knn, (cell, near) = build_nsg_cells(base, R=R, knn_k=k, cells=cells, probe=probe, sample=n, iters=6,
                                           with_knn=True, with_cells=True)
    assert cell.shape == (n,) and near.shape == (cells, probe)
    assert cell.max() < cells
    for c in range(cells):
        nc = near[c]
        assert c not in nc and len(set(nc.tolist())) == probe
    members = [np.nonzero(cell == c)[0] for c in range(cells)]
    bad = 0
    for c in range(cells):
        cand = np.concatenate([members[c]] + [members[j] for j in near[c]])
        cand.sort()
        for a in members[c]:
            others = cand[cand != a]
            dd = _d2(base[a], base[others])
            order = np.lexsort((others, dd))[:k]
            want, wd = others[order], dd[order]
            got = knn[a][knn[a] < n]
            if len(got) == len(want) and np.array_equal(got, want):
                continue
            # equal only up to the order of (nearly) equal distances
            gd = _d2(base[a], base[got])
            if len(got) != len(want) or not np.allclose(np.sort(gd), wd, rtol=1e-9, atol=0):
                bad += 1
    assert bad == 0, bad
    # prune rule on a sample of vertices: walk the k-NN list, keep b unless a
    # kept c is nearer to b than a is
    rng = np.random.default_rng(3)
    for a in rng.choice(n, 200, replace=False):
        kept = []
        for b in knn[a]:
            if b >= n or len(kept) == R:
                break
            dab = _d2(base[a], base[b:b + 1])[0]
            if not kept or not (_d2(base[b], base[np.array(kept)]) < dab).any():
                kept.append(int(b))
        lst = g.nbrs[g.offsets[a]:g.offsets[a + 1]]
        assert list(lst[:len(kept)]) == kept
    # reachability from the entry; entry = nearest to the float64 mean
    seen = np.zeros(n, bool)
    seen[g.entry] = True
    dq = deque([g.entry])
    while dq:
        v = dq.popleft()
        for w in g.nbrs[g.offsets[v]:g.offsets[v + 1]]:
            if not seen[w]:
                seen[w] = True
                dq.append(w)
    assert seen.all()
    mean = base.astype(np.float64).mean(0)
    dm = _d2(mean.astype(np.float64), base)
    assert abs(dm[g.entry] - dm.min()) <= 1e-12 * dm.min()


def test_cell_build_reverse_edges():
    from parallel_anns_b200 import datasets as ds
    from parallel_anns_b200.graph import build_nsg_cells
    n, R = 6000, 12
    base = ds.gaussian_mixture(n, 24, seed=71, means_seed=71)
    g0 = build_nsg_cells(base, R=R, knn_k=16, cells=12, probe=2, sample=n, iters=6)
    g1, knn = build_nsg_cells(base, R=R, knn_k=16, cells=12, probe=2, sample=n, iters=6, reverse=True,
                              with_knn=True)
    assert g1.repaired <= g0.repaired
    lists1 = [g1.nbrs[g1.offsets[a]:g1.offsets[a + 1]] for a in range(n)]
    sets1 = [set(x.tolist()) for x in lists1]
    rng = np.random.default_rng(5)
    for a in rng.choice(n, 300, replace=False):
        kept = []
        for b in knn[a]:
            if b >= n or len(kept) == R:
                break
            dab = _d2(base[a], base[b:b + 1])[0]
            if not kept or not (_d2(base[b], base[np.array(kept)]) < dab).any():
                kept.append(int(b))
        assert list(lists1[a][:len(kept)]) == kept
        for b in kept:
            assert a in sets1[b] or len(lists1[b]) >= R, (a, b)
