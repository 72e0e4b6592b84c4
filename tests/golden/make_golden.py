"""Generate the golden fixtures of the search path from the reference itself.

Run in a container that has the reference sources (its reference binaries are
built by oracle/Makefile into oracle/_ref/):

    python tests/golden/make_golden.py

For each case it writes the inputs (base.fvecs, query.fvecs, graph.nsg,
truenn.bin) and, for every search form listed in CASES, the reference's result
ids (nq x K u32, <form>.ids) and distance-computation count (in
manifest.json). Also the reference's own distances and norms for a fixed set
of (query, vertex) pairs (dist_ip.f32, norms.f32, dist_l2.f32).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from parallel_anns_b200 import datasets as ds  # noqa: E402
from parallel_anns_b200 import formats as fm  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")

# name: (generator, n, d, nq, R)
CASES = {
    "mix3k_d96": ("mixture", 3000, 96, 64, 50),
    "mix1k_d24": ("mixture", 1000, 24, 32, 32),
    "u8_1k_d128": ("uint8", 1000, 128, 32, 64),
}

# (form name, binary, args)
FORMS = [
    ("pss_t1_L100", "ref_pss", dict(K=100, L=100, T=1, X=1)),
    ("pss_t1_L200", "ref_pss", dict(K=100, L=200, T=1, X=4)),
    ("simple_L150", "ref_topm", dict(K=100, L=150, mode="simple")),
    ("topm_M4_L100", "ref_topm", dict(K=100, L=100, M=4, mode="topm_para")),
    ("topm_M16_L200", "ref_topm", dict(K=50, L=200, M=16, mode="topm_seq")),
    ("topm_M64_L100", "ref_topm", dict(K=100, L=100, M=64, mode="topm_para")),
    ("lg_t1_L100", "ref_pss_lg", dict(K=100, L=100, T=1, X=1)),
    ("lg_t1_L250", "ref_pss_lg", dict(K=10, L=250, T=1, X=2)),
    ("efanna_search_L100", "ref_efanna", dict(K=100, L=100, mode="search")),
    ("efanna_opt_L120", "ref_efanna", dict(K=100, L=120, mode="opt")),
]


def make_inputs(kind, n, d, nq, R, out):
    if kind == "mixture":
        base = ds.gaussian_mixture(n, d, seed=11, means_seed=11)
        q = ds.gaussian_mixture(nq, d, seed=12, means_seed=11)
    else:
        base = ds.uint8_cube(n, d, seed=21)
        q = ds.uint8_cube(nq, d, seed=22)
    g = ds.build_nsg_graph(base, R=R, knn_k=64, device="cpu")
    gt_ids, gt_d = ds.ground_truth_fp64_cpu(base, q, 100)
    fm.write_fvecs(os.path.join(out, "base.fvecs"), base)
    fm.write_fvecs(os.path.join(out, "query.fvecs"), q)
    fm.write_nsg(os.path.join(out, "graph.nsg"), g)
    fm.write_true_nn(os.path.join(out, "truenn.bin"), gt_ids, gt_d)
    return base, q, g


def run(binary, out, **kw):
    args = [os.path.join(REF, binary)] + [f"{k}={v}" for k, v in kw.items()] + [f"out={out}"]
    r = subprocess.run(args, check=True, capture_output=True, text=True)
    return json.loads(r.stdout.strip().splitlines()[-1]) if r.stdout.strip() else {}


def main():
    manifest = {}
    for name, (kind, n, d, nq, R) in CASES.items():
        out = os.path.join(HERE, name)
        os.makedirs(out, exist_ok=True)
        base, q, g = make_inputs(kind, n, d, nq, R, out)
        files = dict(data=os.path.join(out, "base.fvecs"), queries=os.path.join(out, "query.fvecs"),
                     nsg=os.path.join(out, "graph.nsg"), truenn=os.path.join(out, "truenn.bin"))
        entry = {"kind": kind, "n": n, "d": d, "nq": nq, "R": R, "width": g.width,
                 "entry": g.entry, "forms": {}}
        for form, binary, kw in FORMS:
            st = run(binary, os.path.join(out, form + ".ids"), **files, **kw)
            entry["forms"][form] = {"binary": binary, "args": kw, "n_dist": st["n_dist"],
                                    "recall100": st["recall100"]}
        ids = np.arange(0, n, max(1, n // 97), dtype=np.uint32)
        ids.tofile(os.path.join(out, "dist_ids.u32"))
        run("ref_pss", os.path.join(out, "dist_ip.f32"), mode="dist",
            ids=os.path.join(out, "dist_ids.u32"), nq=min(nq, 16), **{k: files[k] for k in
                                                                      ("data", "queries", "nsg")})
        os.replace(os.path.join(out, "dist_ip.f32.norms"), os.path.join(out, "norms.f32"))
        run("ref_pss_lg", os.path.join(out, "dist_l2.f32"), mode="dist",
            ids=os.path.join(out, "dist_ids.u32"), nq=min(nq, 16), **{k: files[k] for k in
                                                                      ("data", "queries", "nsg")})
        manifest[name] = entry
        print(name, {f: v["n_dist"] for f, v in entry["forms"].items()})
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
