"""Benchmark workloads: seeded synthetic stand-ins for the reference's datasets.

``batched_fp32_1m``: N = 1,000,000 base vectors, d = 96, from a 64-component
isotropic Gaussian mixture (means ~ N(0, 1), sigma = 0.3), L2-normalised;
queries from the same mixture; NSG-style graph with R = 50 (exact 64-NN,
MRNG prune, medoid entry, reachability repair) built on the GPU by
``graph.build_nsg``; ground truth = top-100 by float64 brute force.

Ground truth: top-100 by float64 brute force (``panns_ground_truth`` on the GPU).
Files are written in the reference's formats (fvecs, .nsg, true-NN) to a cache
directory so that the reference's own binaries can read them and a second
process on the same host reuses them.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

from . import datasets as ds
from . import formats as fm

CACHE = os.environ.get("PANNS_BENCH_CACHE", "/tmp/panns_b200_bench")


def spec_batched_fp32_1m(n=1_000_000, nq=10_000, d=96):
    return {"name": f"mixture64_n{n}_d{d}_q{nq}_R50", "n": n, "d": d, "nq": nq, "R": 50,
            "knn_k": 64, "components": 64, "sigma": 0.3, "base_seed": 1001, "query_seed": 2001,
            "gt_k": 100}


def spec_u8_1m_d128(n=1_000_000, nq=10_000):
    """The reduced-precision config's integer variant: d = 128, components
    uniform in 0..255 stored as uint8 and cast to float32, R = 64."""
    return {"name": f"u8cube_n{n}_d128_q{nq}_R64", "kind": "uint8", "n": n, "d": 128, "nq": nq, "R": 64,
            "knn_k": 64, "base_seed": 1002, "query_seed": 2002, "gt_k": 100}


def spec_mixture_10m_d96(n=10_000_000, nq=10_000):
    """The learned-entry config's base: N = 10M, d = 96, the same mixture
    generator (another seed), R = 50."""
    return {"name": f"mixture64_n{n}_d96_q{nq}_R50", "n": n, "d": 96, "nq": nq, "R": 50,
            "knn_k": 64, "components": 64, "sigma": 0.3, "base_seed": 1003, "query_seed": 2003,
            "gt_k": 100}


def spec_mixture_100m_d96(n=100_000_000, nq=10_000):
    """The large uneven-batch config: N = 100M, d = 96 from a 4,096-component
    mixture (drawn on the GPU), R = 48; graph from exact 64-NN within each of
    10,000 k-means cells and its 3 nearest cells, RNG-pruned to R, reverse
    edges up to R (the mixture's components are tight and far apart, and
    without them a component falls into fragments that only the entry's
    repair links join), medoid entry, repair. Held in memory (no files):
    at this size the reference's loaders would need the whole index twice
    over in host memory."""
    return {"name": f"mixture4096_n{n}_d96_q{nq}_R48", "n": n, "d": 96, "nq": nq, "R": 48, "knn_k": 64,
            "components": 4096, "sigma": 0.3, "base_seed": 1004, "query_seed": 2004, "gt_k": 100,
            "cells": max(1, min(10_000, n // 1000)), "probe": 3, "reverse": True, "reps": 4096, "large": True}


SPECS = {"mixture_1m_d96": spec_batched_fp32_1m, "u8_1m_d128": spec_u8_1m_d128,
         "mixture_10m_d96": spec_mixture_10m_d96, "mixture_100m_d96": spec_mixture_100m_d96}


def describe(spec) -> str:
    """One line naming the workload with its sizes."""
    if spec.get("kind") == "uint8":
        data = f"{spec['n'] // 1000}k x {spec['d']}d integer-valued (uniform 0..255, uint8 cast to float32)"
    else:
        data = (f"{spec['n'] // 1000}k x {spec['d']}d mixture{spec['components']} "
                f"(sigma {spec['sigma']}, unit norm)")
    return f"{data}, NSG-style graph R={spec['R']}, {spec['nq']} queries, K={spec['gt_k']}"


def vectors(spec, count, seed):
    """`count` vectors of the workload's distribution (queries use the base's
    mixture means)."""
    if spec.get("kind") == "uint8":
        return ds.uint8_cube(count, spec["d"], seed=seed)
    if spec.get("large"):
        return ds.gaussian_mixture_gpu(count, spec["d"], spec["components"], spec["sigma"], seed=seed,
                                       means_seed=spec["base_seed"])
    return ds.gaussian_mixture(count, spec["d"], spec["components"], spec["sigma"], seed=seed,
                               means_seed=spec["base_seed"])


def paths(spec):
    root = os.path.join(CACHE, spec["name"])
    return {k: os.path.join(root, v) for k, v in
            dict(root="", base="base.fvecs", query="query.fvecs", graph="graph.nsg",
                 truenn="truenn.bin", meta="meta.json").items()}


def cached(spec) -> bool:
    """True when the cache holds this exact workload."""
    p = paths(spec)
    if not os.path.exists(p["meta"]):
        return False
    with open(p["meta"]) as f:
        return json.load(f).get("spec") == spec


def build(spec, device=None, log=print):
    """Build (or load from the cache) a workload; returns a dict of arrays + paths."""
    if cached(spec):
        return load(spec)
    t0 = time.time()
    base = vectors(spec, spec["n"], spec["base_seed"])
    q = vectors(spec, spec["nq"], spec["query_seed"])
    t1 = time.time()
    g = build_graph(base, spec, device)
    t2 = time.time()
    gt_ids, gt_d = ground_truth(base, g, q, spec["gt_k"], device)
    t3 = time.time()
    import torch
    built_by = "gpu (graph_build.cu, gt_kernel.cuh)" if torch.cuda.is_available() else "torch on the host"
    return store(spec, base, q, g, gt_ids, gt_d, built_by,
                 {"generate": t1 - t0, "graph": t2 - t1, "ground_truth": t3 - t2}, log=log)


def store(spec, base, q, g, gt_ids, gt_d, built_by, build_s, log=print):
    """Write a built workload to the cache in the reference's formats (fvecs,
    .nsg, true-NN) with its meta record; returns the workload dict."""
    p = paths(spec)
    os.makedirs(p["root"], exist_ok=True)
    fm.write_fvecs(p["base"], base)
    fm.write_fvecs(p["query"], q)
    fm.write_nsg(p["graph"], g)
    fm.write_true_nn(p["truenn"], gt_ids, np.asarray(gt_d).astype(np.float32))
    meta = {"spec": spec, "width": g.width, "entry": g.entry, "avg_degree": float(g.nbrs.size / g.n),
            "built_by": built_by, "build_s": build_s}
    with open(p["meta"], "w") as f:
        json.dump(meta, f)
    if log:
        log(f"workload {spec['name']}: built by {built_by} in {sum(build_s.values()):.1f}s {build_s}")
    return {"base": base, "queries": q, "graph": g, "gt": gt_ids, "paths": p, "meta": meta}


def build_graph(base, spec, device=None):
    """The workload's graph: the library's GPU construction (include/panns_build.h)
    when a GPU is present, else the torch restatement in datasets.py (same rule)."""
    import torch
    if torch.cuda.is_available():
        from .graph import build_nsg, build_nsg_cells
        dev = torch.device(device) if device is not None else torch.device("cuda", 0)
        if spec.get("cells"):
            return build_nsg_cells(base, R=spec["R"], knn_k=spec["knn_k"], cells=spec["cells"], probe=spec["probe"],
                                   sample=min(spec["n"], 2_000_000), iters=10, seed=1, device=dev.index or 0,
                                   reverse=spec.get("reverse", False))
        return build_nsg(base, R=spec["R"], knn_k=spec["knn_k"], device=dev.index or 0)
    return ds.build_nsg_graph(base, R=spec["R"], knn_k=spec["knn_k"], device="cpu")


def ground_truth(base, graph, queries, k, device=None):
    """Top-k by float64 brute force: the library's GPU kernel when a GPU is
    present (panns_ground_truth), else torch float64 on the CPU."""
    import torch
    if torch.cuda.is_available():
        from .searching import Index, ground_truth as gpu_gt
        dev = torch.device(device) if device is not None else torch.device("cuda", 0)
        with Index(dev.index or 0) as ix:
            ix.set_base(base)
            ix.set_graph(graph)
            return gpu_gt(ix, queries, k)
    return ds.exact_knn(base, queries, k, device="cpu", dtype=torch.float64, block=512)


def load(spec):
    p = paths(spec)
    with open(p["meta"]) as f:
        meta = json.load(f)
    return {"base": fm.read_fvecs(p["base"]), "queries": fm.read_fvecs(p["query"]),
            "graph": fm.read_nsg(p["graph"]), "gt": fm.read_true_nn(p["truenn"])[0], "paths": p,
            "meta": meta}


def tuning_set(spec, W, n_tune=10_000, device=None):
    """Held-out queries (same mixture, another seed) with their float64 top-100,
    for choosing operating points without looking at the evaluated queries."""
    path = os.path.join(paths(spec)["root"], f"tune_q{n_tune}.npz")
    if os.path.exists(path):
        z = np.load(path)
        return z["q"], z["gt"]
    q = vectors(spec, n_tune, spec["query_seed"] + 1)
    gt, _ = ground_truth(W["base"], W["graph"], q, spec["gt_k"], device)
    np.savez(path, q=q, gt=gt)
    return q, gt


def learned_model(spec, index, n_train=200_000, R=1024, log=print):
    """The entry / L-budget network for this workload, trained on n_train
    held-out queries (cached next to the workload)."""
    from . import learned as LE
    cache = os.path.join(paths(spec)["root"], f"learned_R{R}_t{n_train}.npz")
    train_q = vectors(spec, n_train, spec["base_seed"] + 2000)
    t0 = time.time()
    m = LE.build_model(index, train_q, R=R, K=spec["gt_k"], M=8, L_ref=1000, T=10, epochs=10, batch=1024,
                       lr=2e-3, lam=1.0, seed=0, kmeans_iters=15, cache=cache, log=log)
    if log:
        log(f"learned model ready in {time.time() - t0:.1f}s ({cache})")
    return m
