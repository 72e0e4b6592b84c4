"""efanna2e's IndexNSG::Build (include/efanna2e/index_nsg.cpp:403-450) on the
GPU, against the reference's own build (tools/test_nsg_index.cpp, one OpenMP
thread): the .nsg files must be equal byte for byte.

* the committed fixture (tests/golden/efanna_build, made by
  tests/golden/make_efanna_build.py): rand() init ids for every vertex,
  findroot repairs and a width above R;
* fresh seeded cases run through oracle/_ref/ref_nsg_build in the test: the
  first L of the navigating node's k-NN list as init ids (L <= k), d = 96 and
  d = 24 (the reference's lane order with d % 16 == 8), a prune limited by C.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def build_bytes(base, knn, L, R, C, path):
    from parallel_anns_b200 import formats as fm
    from parallel_anns_b200.graph import efanna_build
    g = efanna_build(base, knn, L, R, C)
    fm.write_nsg(path, g)
    with open(path, "rb") as f:
        return f.read(), g


def test_efanna_build_matches_reference_fixture(tmp_path):
    from parallel_anns_b200 import formats as fm
    d = os.path.join(GOLDEN, "efanna_build")
    with open(os.path.join(d, "case.json")) as f:
        c = json.load(f)
    base = fm.read_fvecs(os.path.join(d, "base.fvecs"))
    knn = O.read_efanna_knn(os.path.join(d, "knn.graph"))
    got, g = build_bytes(base, knn, c["L"], c["R"], c["C"], str(tmp_path / "gpu.nsg"))
    with open(os.path.join(d, "ref.nsg"), "rb") as f:
        ref = f.read()
    assert g.width > c["R"] and c["new_roots"] > 0  # the repair path ran
    assert got == ref


@pytest.mark.parametrize("n,d,k,L,R,C,seed", [
    (3000, 96, 50, 40, 32, 200, 91),
    (2500, 24, 32, 32, 16, 64, 92),
    (2000, 96, 24, 48, 12, 150, 93),
])
def test_efanna_build_matches_reference_binary(tmp_path, n, d, k, L, R, C, seed):
    if not os.path.exists(O.ref_binary("ref_nsg_build")):
        pytest.skip("oracle/_ref/ref_nsg_build not built")
    from parallel_anns_b200 import datasets as ds
    from parallel_anns_b200 import formats as fm
    base = ds.gaussian_mixture(n, d, seed=seed, means_seed=seed)
    knn, _ = O.host_knn(base, None, k)
    bp, kp, rp = str(tmp_path / "b.fvecs"), str(tmp_path / "k.graph"), str(tmp_path / "ref.nsg")
    fm.write_fvecs(bp, base)
    O.write_efanna_knn(kp, knn)
    O.ref_nsg_build(bp, kp, L, R, C, rp, threads=1)
    got, _ = build_bytes(base, knn, L, R, C, str(tmp_path / "gpu.nsg"))
    with open(rp, "rb") as f:
        assert got == f.read()


def test_efanna_build_rejects_bad_input():
    from parallel_anns_b200 import native as N
    from parallel_anns_b200.graph import efanna_build
    base = np.zeros((100, 20), np.float32)  # d not a multiple of 8
    with pytest.raises(N.PannsError):
        efanna_build(base, np.zeros((100, 4), np.uint32), 10, 4, 20)
    base = np.zeros((100, 16), np.float32)
    with pytest.raises(N.PannsError):
        efanna_build(base, np.full((100, 4), 100, np.uint32), 10, 4, 20)  # id >= n
