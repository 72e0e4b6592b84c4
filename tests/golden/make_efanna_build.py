"""Writes the efanna2e Build fixture (test infrastructure): a seeded
2,000 x 32 mixture, its exact 20-NN graph in EFANNA's file layout, and the
.nsg graph that the reference's own tools/test_nsg_index.cpp (built unchanged
as oracle/_ref/ref_nsg_build) makes from them with L = 30, R = 6, C = 60 at
one OpenMP thread. L > k makes every vertex draw rand() ids, and R = 6 leaves
vertices the first depth-first walk does not reach, so the fixture also
covers findroot and the width update of tree_grow.

    python tests/golden/make_efanna_build.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from parallel_anns_b200 import datasets as ds  # noqa: E402
from parallel_anns_b200 import formats as fm  # noqa: E402

CASE = dict(n=2000, d=32, k=20, L=30, R=6, C=60, seed=84)


def main():
    out = os.path.join(HERE, "efanna_build")
    os.makedirs(out, exist_ok=True)
    c = CASE
    base = ds.gaussian_mixture(c["n"], c["d"], seed=c["seed"], means_seed=c["seed"])
    knn, _ = O.host_knn(base, None, c["k"])
    fm.write_fvecs(os.path.join(out, "base.fvecs"), base)
    O.write_efanna_knn(os.path.join(out, "knn.graph"), knn)
    log = O.ref_nsg_build(os.path.join(out, "base.fvecs"), os.path.join(out, "knn.graph"), c["L"], c["R"], c["C"],
                          os.path.join(out, "ref.nsg"), threads=1)
    with open(os.path.join(out, "case.json"), "w") as f:
        json.dump(dict(c, new_roots=log.count("new root")), f)


if __name__ == "__main__":
    main()
