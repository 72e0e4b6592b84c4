#!/usr/bin/env python
"""Benchmark of the batched best-first NSG search on B200.

Workload (batched FP32): N = 1,000,000 base vectors, d = 96, 64-component
Gaussian mixture (sigma 0.3, unit norm), NSG-style graph R = 50; 10,000
evaluation queries per GPU (weak scaling: rank r searches its own 10,000);
K = 100. Metric: queries per second at recall@100 >= 0.95.

Operating points are chosen by the autotuner (parallel_anns_b200/autotune.py)
on 10,000 held-out tuning queries of another seed, never on the evaluated
ones: per candidate (storage FP32 / BF16 / FP8, with or without the learned
entry network, M) the smallest L reaching the target, then the warps per
block; the fastest wins ("value"), and the plain FP32 search is tuned and
reported beside it ("plain_fp32"). The learned network is trained on the GPU
on 200,000 held-out queries before tuning (cached with the workload).

One step = one batched search of all of a rank's queries (one kernel launch).
``value``: device time of the search kernel (CUDA events) with base, graph
and queries resident in HBM; the 384 MB base set alone is larger than L2 and
L2 is also flushed (a 256 MB write) before every step.
``e2e``: the same search through the C ABI's host-pointer entry point
(panns_search_host: queries copied host->device from pinned memory, ids copied
back into pinned memory), wall time per step.
``batching``: batches of 1, 64 and 1,000 queries back to back through the
asynchronous device-pointer entry point with the CUDA-graph-captured launch.

``--impl reference`` times the reference's own PSS_v5
(core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp, built from its
sources into oracle/_ref/ref_pss) on all host cores, on a bounded query sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "QPS at recall@100>=0.95, 1M x 96d; learned+BF16 vs plain FP32 GPU vs CPU"
UNIT = "queries/s"
RECALL_TARGET = 0.95
# Operating points are tuned on held-out queries to the target plus a margin
# (about three standard errors of a 10,000-query recall estimate), so that the
# evaluated queries meet the target too.
TUNE_TARGET = RECALL_TARGET + 0.002
L_SWEEP = [100, 128, 160, 200, 256, 320, 400, 512, 640, 800]
M_SWEEP = [1, 2, 4, 8, 16]


def metric_for(spec):
    """The metric's name for a workload (the default one is the name the
    benchmark is quoted under)."""
    if spec["n"] == 1_000_000 and spec["d"] == 96:
        return METRIC
    return METRIC.replace("1M x 96d", f"{spec['n'] / 1e6:g}M x {spec['d']}d")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def nproc():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference_pss(paths, nq, L, T, X=1, reps=1, K=100, timeout=900, binary="ref_pss", inner=None):
    """The reference's PSS_v5 binaries on the cached files: ref_pss (intra-query,
    T threads per query) or ref_multi (inter-query: T / inner queries at a time,
    `inner` threads each)."""
    exe = os.path.join(ROOT, "oracle", "_ref", binary)
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    env = dict(os.environ, OMP_PROC_BIND="close", OMP_PLACES="cores")
    with tempfile.TemporaryDirectory() as tmp:
        args = [exe, f"data={paths['base']}", f"queries={paths['query']}", f"nsg={paths['graph']}",
                f"truenn={paths['truenn']}", f"K={K}", f"L={L}", f"T={T}", f"X={X}", f"nq={nq}",
                f"reps={reps}", f"out={os.path.join(tmp, 'ids.bin')}"]
        if inner is not None:
            args.append(f"inner={inner}")
        r = subprocess.run(args, check=True, capture_output=True, text=True, env=env, timeout=timeout)
    return json.loads(r.stdout.strip().splitlines()[-1])


# The reference's CPU modes timed as baselines: (name, binary, X, inner).
REF_MODES = [("PSS_v5 intra-query", "ref_pss", 1, None), ("PSS_v5 intra-query", "ref_pss", 4, None),
             ("PSS_v5 inter-query (multi_queries_LG, 1 thread per query)", "ref_multi", 1, 1)]


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def host_workload(spec, log):
    """The workload's inputs built on the host CPU without the GPU library:
    vectors from the same seeded generator, then the graph and the float64
    ground truth by oracle/host_build.c (exact: the same graph as the GPU
    construction and the same top-k as a float64 brute force). The
    reference arm uses this, so its process never maps the library."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from parallel_anns_b200 import workloads
    t0 = time.time()
    base = workloads.vectors(spec, spec["n"], spec["base_seed"])
    q = workloads.vectors(spec, spec["nq"], spec["query_seed"])
    t1 = time.time()
    g, _ = O.host_build_nsg(base, spec["knn_k"], spec["R"])
    t2 = time.time()
    gt_ids, gt_d = O.host_knn(base, q, spec["gt_k"])
    t3 = time.time()
    return workloads.store(spec, base, q, g, gt_ids, gt_d, HOST_BUILT,
                           {"generate": t1 - t0, "graph": t2 - t1, "ground_truth": t3 - t2}, log=log)


HOST_BUILT = "host CPU (oracle/host_build.c)"


def check_host_inputs(W, spec, local, log):
    """When the cached inputs were built on the host, rebuild the graph and the
    ground truth on the GPU and compare them byte for byte."""
    import numpy as np
    from parallel_anns_b200 import workloads
    from parallel_anns_b200.graph import build_nsg
    built_by = W["meta"].get("built_by", "gpu")
    out = {"built_by": built_by}
    if built_by != HOST_BUILT:
        return out
    g, h = build_nsg(W["base"], R=spec["R"], knn_k=spec["knn_k"], device=local), W["graph"]
    same_g = (g.entry == h.entry and g.width == h.width and np.array_equal(g.offsets, h.offsets)
              and np.array_equal(g.nbrs, h.nbrs))
    gt, _ = workloads.ground_truth(W["base"], h, W["queries"], spec["gt_k"], f"cuda:{local}")
    same_gt = bool(np.array_equal(gt, W["gt"]))
    out["gpu_rebuild_identical"] = bool(same_g and same_gt)
    if not out["gpu_rebuild_identical"]:
        log(f"inputs: GPU rebuild differs from the host-built files (graph {same_g}, ground truth {same_gt})")
    return out


def parity_sample(index, choice, paths, K, nq_sample, log):
    """Ids of the exact FP32 search at the plain operating point against the
    reference's own top-M search at one thread (oracle/_ref/ref_topm: the
    sequential search for M = 1, para_search_with_top_m_pure otherwise) on the
    first nq_sample evaluation queries: rows equal, distance counts equal."""
    import numpy as np
    from parallel_anns_b200 import native as N
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_topm")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ref_topm not built"}
    mode = "simple" if choice.M == 1 else "topm_para"
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "ids.bin")
        r = subprocess.run([exe, f"data={paths['base']}", f"queries={paths['query']}", f"nsg={paths['graph']}",
                            f"K={K}", f"L={choice.L}", f"M={choice.M}", f"mode={mode}", "T=1",
                            f"nq={nq_sample}", f"out={out}"], check=True, capture_output=True, text=True,
                           timeout=900)
        ref = np.fromfile(out, dtype=np.uint32).reshape(-1, K)
    st_ref = json.loads(r.stdout.strip().splitlines()[-1])
    kw = dict(choice.search_kwargs(), storage=N.STORE_FP32, flags=0)
    ids, st = index.search(K=K, q_begin=0, nq=nq_sample, distance=N.DIST_NORM_IP, **kw)
    rows_equal = int((ids == ref).all(1).sum())
    res = {"queries": nq_sample, "rows_equal": rows_equal, "n_dist_equal": int(st["n_dist"]) == int(st_ref["n_dist"]),
           "n_dist": int(st["n_dist"]), "reference": f"ref_topm {mode} T=1 L={choice.L} M={choice.M}"}
    log(f"parity sample: {res}")
    return res


# ---------------------------------------------------------------------------
def bench_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from parallel_anns_b200 import autotune as AT
    from parallel_anns_b200 import learned as LE
    from parallel_anns_b200 import native as N
    from parallel_anns_b200 import workloads
    from parallel_anns_b200.replicas import Ranks, shard
    from parallel_anns_b200.searching import Index, recall

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900),
                                device_id=torch.device("cuda", local))
    ranks = Ranks(world, device="cuda")
    barrier = ranks.barrier
    max_over_ranks = ranks.max

    spec = workloads.SPECS[args.workload](**({"n": args.n} if args.n else {}), nq=args.nq * world)
    args.n = spec["n"]
    if spec.get("large"):
        if world > 1:
            raise SystemExit(f"workload {args.workload}: one GPU only (the whole index on each replica)")
        return bench_large(args, spec)
    fixed = bool(args.L and args.M)  # a given operating point: no tuning set, no autotuning
    if rank == 0:
        W = workloads.build(spec, device=f"cuda:{local}", log=log)
        if not fixed:
            tune_q, tune_gt = workloads.tuning_set(spec, W, device=f"cuda:{local}")
    barrier()
    if rank != 0:
        W = workloads.load(spec)
        if not fixed:
            tune_q, tune_gt = workloads.tuning_set(spec, W)
    inputs = check_host_inputs(W, spec, local, log) if rank == 0 else None
    q_all, gt_all = W["queries"], W["gt"]
    qs = np.ascontiguousarray(q_all[shard(rank, args.nq)])
    gts = gt_all[shard(rank, args.nq)]
    nq, d, K = qs.shape[0], qs.shape[1], 100

    # One handle with the BF16 copy (its float32 rows serve the exact search),
    # one with the FP8 copy.
    handles = {}
    for store in (N.STORE_BF16, N.STORE_FP8):
        ix = Index(local)
        ix.set_base(W["base"], storage=store)
        ix.set_graph(W["graph"])
        ix.set_queries(qs)
        handles[store] = ix
    handles[N.STORE_FP32] = handles[N.STORE_BF16]
    names = {N.STORE_FP32: "fp32", N.STORE_BF16: "bf16", N.STORE_FP8: "fp8"}

    # The learned entry / L-budget network (trained on the GPU on held-out
    # queries; rank 0 builds it, the others load the cached file).
    model = None
    if not args.no_learned and (not fixed or args.entries):
        if rank == 0:
            model = workloads.learned_model(spec, handles[N.STORE_BF16], log=log)
        barrier()
        if rank != 0:
            model = workloads.learned_model(spec, handles[N.STORE_BF16], log=None)
    # Learned options: entries with a few plain init ids kept, entries only, and
    # entries with the plain search for queries the network is unsure of.
    learned_opts = [dict(E=8, L_init=8, use_L=False), dict(E=32, L_init=0, use_L=False),
                    dict(E=16, L_init=16, use_L=False, min_conf=0.5)]

    # Operating points, chosen by the autotuner on the tuning queries (not the
    # evaluated ones) on rank 0: the plain FP32 search, and the fastest of all
    # storages with and without the network.
    Ms = [args.M] if args.M else M_SWEEP
    stores = [args.storage] if args.storage is not None else [N.STORE_FP32, N.STORE_BF16, N.STORE_FP8]
    choices = None
    if fixed:
        c = {"storage": args.storage or 0, "M": args.M, "L": args.L, "warps_per_block": args.wpb,
             "learned": None, "blocks_per_sm": 0, "warps_per_query": 1}
        if args.entries:
            parts = args.entries.split(":")
            c["learned"] = {"E": int(parts[0]), "L_init": int(parts[1]), "use_L": False}
            if len(parts) > 2:
                c["learned"]["min_conf"] = float(parts[2])
        choices = {"plain": dict(c, storage=0, learned=None), "head": c, "tables": []}
    elif rank == 0:
        t0 = time.time()
        plain = AT.tune(handles[N.STORE_FP32], tune_q, tune_gt, K=K, target=TUNE_TARGET,
                        storages=(N.STORE_FP32,), Ms=Ms, wpbs=(2, 4), wpqs=(1, 2, 4, 8))
        cands = [plain]
        for store in stores:
            if store == N.STORE_FP32 and model is None:
                continue
            c = AT.tune(handles[store], tune_q, tune_gt, K=K, target=TUNE_TARGET, storages=(store,), Ms=Ms,
                        wpbs=(2, 4), wpqs=(1, 2, 4, 8), learned_model=model,
                        learned_opts=learned_opts if model is not None else (),
                        include_plain=store != N.STORE_FP32)
            cands.append(c)
        head = min(cands, key=lambda c: c.kernel_ms)
        log(f"autotune {time.time() - t0:.1f}s: plain fp32 {plain.L}/{plain.M}/{plain.warps_per_block} "
            f"{plain.kernel_ms:.3f} ms; head {names[head.storage]} L={head.L} M={head.M} "
            f"w={head.warps_per_block} learned={head.learned} {head.kernel_ms:.3f} ms")
        strip = lambda c: {k: v for k, v in c.__dict__.items() if k != "table"}
        choices = {"plain": strip(plain), "head": strip(head),
                   "tables": [r for c in cands for r in c.table]}
    choices = ranks.broadcast_json(choices, 0)
    plain = AT.Choice(**choices["plain"])
    head = AT.Choice(**choices["head"])
    if head.learned is not None:
        LE.attach(handles[head.storage], model, **head.learned)

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    sampler = ClockSampler(local)

    def run(c):
        return handles[c.storage].search(K=K, distance=N.DIST_NORM_IP, **c.search_kwargs())

    def timed(c):
        for _ in range(args.warmup):
            run(c)
        barrier()
        torch.cuda.synchronize()
        kms = 0.0
        tot_ = {"n_dist": 0, "n_edges": 0, "n_expand": 0, "n_iter": 0}
        ids_ = None
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ids_, st = run(c)
            kms += st["kernel_ms"]
            for k in tot_:
                tot_[k] += st[k]
        barrier()
        torch.cuda.synchronize()
        return kms, tot_, ids_

    sampler.start()
    kernel_ms, tot, last_ids = timed(head)
    kernel_ms_max = max_over_ranks(kernel_ms)
    rec = recall(last_ids, gts, 100, 100)
    learned_info = None
    if head.learned is not None:
        Lq, fb, _ = LE.record(handles[head.storage], nq)
        learned_info = {"options": head.learned, "fallback_rate": round(float(fb.mean()), 4),
                        "mean_L": round(float(Lq.mean()), 1), "R": model.R,
                        "training_queries": 200_000}
    if (plain.storage, plain.L, plain.M, plain.learned, plain.warps_per_block, plain.warps_per_query,
            plain.blocks_per_sm) == (head.storage, head.L, head.M, head.learned, head.warps_per_block,
                                     head.warps_per_query, head.blocks_per_sm):
        p_ms, p_ids, p_tot = kernel_ms, last_ids, tot
    else:
        p_ms, p_tot, p_ids = timed(plain)
        if head.learned is not None:  # timed(plain) ran without the flag; the network stays attached
            pass
    p_ms_max = max_over_ranks(p_ms)
    p_rec = recall(p_ids, gts, 100, 100)

    # End to end through the host-pointer C ABI call, queries and ids in pinned
    # host memory; the L2 flush between steps is outside the timed spans.
    ixh = handles[head.storage]
    kw = head.search_kwargs()
    q_pin = torch.from_numpy(qs).pin_memory().numpy()
    out_pin = torch.empty((nq, K), dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    for _ in range(args.warmup):
        ixh.search(q_pin, K=K, out=out_pin, **kw)
    barrier()
    torch.cuda.synchronize()
    e2e_s = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ids_e2e, st_e2e = ixh.search(q_pin, K=K, out=out_pin, **kw)
        e2e_s += time.perf_counter() - t0
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(e2e_s)
    clocks = sampler.stop()
    assert np.array_equal(ids_e2e, last_ids)

    # Batch sizes 1, 64 and 1000 through the asynchronous device-pointer entry
    # point with the CUDA-graph-captured launch, batches back to back on one
    # stream (device time from the first launch to the last result).
    # Per batch size the warps per query is tuned too (1, 2, 4), at the head's L and M.
    batching = {}
    qd = torch.from_numpy(qs).cuda()
    stream = torch.cuda.Stream()
    for B, nb in ((1, 300), (64, 60), (1000, 10)):
        outb = torch.empty((B, K), dtype=torch.int32, device="cuda")
        best_b, tried = None, {}
        # the head's own configuration, then the head's storage, L and M
        # without the learned network, with 1, 2 and 4 warps per query
        options = [(head.warps_per_query, ixh, dict(kw, flags=kw["flags"] | N.FLAG_CUDA_GRAPH))]
        for wq in (1, 2, 4, 8):
            if wq == head.warps_per_query and head.learned is None:
                continue  # the head itself
            options.append((wq, ixh, dict(kw, flags=N.FLAG_CUDA_GRAPH, warps_per_query=wq)))
            if head.learned is not None and wq != head.warps_per_query:  # the network with several warps
                options.append((wq, ixh, dict(kw, flags=kw["flags"] | N.FLAG_CUDA_GRAPH, warps_per_query=wq)))
        if head.storage != N.STORE_FP32:  # and the float32 rows with several warps
            for wq in (2, 4, 8):
                options.append((wq, handles[N.STORE_FP32],
                                dict(kw, storage=N.STORE_FP32, flags=N.FLAG_CUDA_GRAPH, warps_per_query=wq)))
        for wq, ixb, kwb in options:
            for i in range(3):
                ixb.search_device(qd[i * B:(i + 1) * B], outb, K=K, stream=stream, **kwb)
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for i in range(nb):
                s0 = (i * B) % (nq - B + 1)
                ixb.search_device(qd[s0:s0 + B], outb, K=K, stream=stream, **kwb)
            e1.record(stream)
            stream.synchronize()
            ms = e0.elapsed_time(e1)
            r_ = {"qps": round(nb * B / (ms / 1e3), 1), "ms_per_batch": round(ms / nb, 4), "warps_per_query": wq,
                  "storage": names[kwb["storage"]]}
            r_["learned"] = bool(kwb["flags"] & N.FLAG_LEARNED)
            tried[f"{wq}/{names[kwb['storage']]}" + ("+learned" if r_["learned"] else "")] = r_["qps"]
            if best_b is None or r_["qps"] > best_b["qps"]:
                best_b = r_
        batching[str(B)] = dict(best_b, qps_by_warps_per_query=tried)
    batching[str(nq)] = {"qps": round(nq * args.steps / (kernel_ms / 1e3), 1),
                         "ms_per_batch": round(kernel_ms / args.steps, 4)}

    # Distance error of the returned ids against float64 (reduced storage re-ranks in float32).
    ids64 = last_ids[: min(200, nq)].astype(np.int64)
    qq = qs[: ids64.shape[0]].astype(np.float64)
    d64 = ((W["base"][ids64].astype(np.float64) - qq[:, None, :]) ** 2).sum(-1)
    g64 = ((W["base"][gts[: ids64.shape[0], :K].astype(np.int64)].astype(np.float64) - qq[:, None, :]) ** 2).sum(-1)
    dist_err = float(np.mean(np.abs(np.sort(d64, 1) - np.sort(g64, 1)) / np.maximum(np.sort(g64, 1), 1e-12)))

    # Roofline of the search kernel: algorithmic bytes per launch
    # = n_dist * (s*d + 4 norm) + 4 * sum(1 + degree) over expansions + nq * (4d + 4K)
    #   (+ nq * L * (4d + 4) for the float32 re-rank of a reduced copy).
    steps = args.steps
    store, L, M = head.storage, head.L, head.M
    s_el = {N.STORE_FP32: 4, N.STORE_BF16: 2, N.STORE_FP8: 1}[store]
    alg_bytes = (tot["n_dist"] * (s_el * d + 4) + 4 * tot["n_edges"]) / steps + nq * (4 * d + 4 * K)
    if store != N.STORE_FP32:
        alg_bytes += nq * L * (4 * d + 4)
    launch_s = kernel_ms / steps / 1e3
    achieved = alg_bytes / launch_s / 1e9
    peak, peak_kind = measured_peak_hbm()
    traffic = None
    tp = os.path.join(ROOT, "profiles", "search_kernel_traffic.json")
    if os.path.exists(tp):
        try:
            with open(tp) as f:
                entries = json.load(f)
            for tj in entries if isinstance(entries, list) else [entries]:
                if (tj.get("L"), tj.get("M"), tj.get("n"), tj.get("storage"), tj.get("learned"),
                        tj.get("warps_per_query", 1)) == (L, M, args.n, names[store], head.learned is not None,
                                                          head.warps_per_query):
                    traffic = tj["dram_bytes_per_query"] * nq
        except Exception:
            traffic = None
    p_alg = (p_tot["n_dist"] * (4 * d + 4) + 4 * p_tot["n_edges"]) / steps + nq * (4 * d + 4 * K)

    total_q = nq * world * steps
    value = total_q / (kernel_ms_max / 1e3)
    e2e_value = total_q / e2e_s

    cpu_base, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_base = cpu_baseline(W["paths"], plain.L, nq, log)
    if rank == 0 and not args.no_parity:
        try:
            parity = parity_sample(handles[N.STORE_FP32], plain, W["paths"], K, min(500, nq), log)
        except Exception as e:  # reported, never fatal
            parity = {"unavailable": str(e)[:200]}

    if world > 1:
        dist.barrier()
    if rank == 0:
        details = {"autotune": choices["tables"], "batching": batching, "cpu_baseline": cpu_base,
                   "learned": learned_info, "inputs": inputs}
        log("details " + json.dumps(details))
        # The JSON line stays short (the full tables go to stderr above).
        line = {
            "metric": metric_for(spec), "value": round(value, 1), "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": args.warmup,
            "ms_per_step": round(kernel_ms_max / steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": names[store], "data": "synthetic",
            "config": {"workload": "batched search, " + workloads.describe(spec) + " (per GPU)",
                       "L": L, "M": M, "warps_per_block": head.warps_per_block,
                       "warps_per_query": head.warps_per_query, "blocks_per_sm": head.blocks_per_sm,
                       "storage": names[store], "accumulate": "f32",
                       "rerank": "exact f32 of the final L" if store != N.STORE_FP32 else None,
                       "learned": None if learned_info is None else learned_info["options"],
                       "mode": "NSG_SEQ" if M == 1 else "TOP_M", "distance": "NORM_IP",
                       "recall100": round(rec, 5), "rel_dist_err_vs_fp64": float(f"{dist_err:.3g}"),
                       "parallelism": f"replicas x{world}",
                       "operating_point": "fixed by --L/--M" if fixed else "autotuned on 10k held-out queries",
                       "l2": "inputs > L2 and a 256 MB L2 flush before each step",
                       "inputs": inputs},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind},
            "e2e": {"value": round(e2e_value, 1), "unit": UNIT,
                    "h2d_bytes_per_step": nq * d * 4,
                    "d2h_bytes_per_step": nq * K * 4 + nq * 16 + 4},
            "gpu_launches": steps,
            "plain_fp32": {"value": round(nq * world * steps / (p_ms_max / 1e3), 1),
                           "L": plain.L, "M": plain.M, "warps_per_query": plain.warps_per_query,
                           "recall100": round(p_rec, 5),
                           "roofline_frac": round(p_alg / (p_ms / steps / 1e3) / 1e9 / peak, 4)},
            "parity": parity,
            "batching_qps": {b: v["qps"] for b, v in batching.items()},
            "clocks": clocks,
            "cpu_baseline": None if cpu_base is None else {k: v for k, v in cpu_base.items() if k != "modes"},
        }
        print(json.dumps(line), flush=True)
    for ixx in set(handles.values()):
        ixx.close()
    if world > 1:
        dist.destroy_process_group()


def bench_large(args, spec):
    """The large uneven-batch configuration on one GPU, held in memory: base
    drawn on the GPU, the cell-restricted graph, one handle with the float32
    rows and a BF16 copy, float64 ground truth, the learned network, the
    autotuner's head (BF16 +- network) against plain FP32, then batches of
    1 ... 65,536 queries at the head's configuration and at L = 200 and 400."""
    import numpy as np
    import torch

    from parallel_anns_b200 import autotune as AT
    from parallel_anns_b200 import learned as LE
    from parallel_anns_b200 import native as N
    from parallel_anns_b200 import workloads
    from parallel_anns_b200.searching import Index, ground_truth as gpu_gt, recall

    K, nq, d = 100, args.nq, spec["d"]
    tm = {}
    t0 = time.time()
    base = workloads.vectors(spec, spec["n"], spec["base_seed"])
    qs = workloads.vectors(spec, nq, spec["query_seed"])
    tune_q = workloads.vectors(spec, 10_000, spec["query_seed"] + 1)
    tm["generate_s"] = round(time.time() - t0, 1)
    t0 = time.time()
    g = workloads.build_graph(base, spec)
    tm["graph_s"] = round(time.time() - t0, 1)
    ginfo = {"entry": int(g.entry), "width": int(g.width), "avg_degree": round(g.nbrs.size / g.n, 2),
             "repaired": int(getattr(g, "repaired", 0)), "cells": spec["cells"], "probe": spec["probe"]}
    log(f"graph: {ginfo} in {tm['graph_s']} s")
    t0 = time.time()
    ix = Index(0)
    ix.set_base(base, storage=N.STORE_BF16)
    ix.set_graph(g)
    del g
    ix.set_queries(qs)
    gts, _ = gpu_gt(ix, qs, K)
    tune_gt, _ = gpu_gt(ix, tune_q, K)
    tm["index_and_ground_truth_s"] = round(time.time() - t0, 1)
    model = None
    if not args.no_learned:
        t0 = time.time()
        # One representative per mixture component, and trace labels from a
        # queue long enough to hold every neighbour of the entry (the
        # components meet only there).
        model = LE.build_model(ix, workloads.vectors(spec, 200_000, spec["base_seed"] + 2000), R=spec["reps"],
                               K=K, M=8, L_ref=max(1000, ginfo["width"] + 1000), T=10, epochs=10, batch=1024,
                               lr=2e-3, lam=1.0, seed=0, kmeans_iters=8, log=log)
        tm["learned_s"] = round(time.time() - t0, 1)
    learned_opts = [dict(E=8, L_init=8, use_L=False), dict(E=16, L_init=16, use_L=False, min_conf=0.5)]
    t0 = time.time()
    Ms = [args.M] if args.M else M_SWEEP
    plain = AT.tune(ix, tune_q, tune_gt, K=K, target=TUNE_TARGET, storages=(N.STORE_FP32,), Ms=Ms, wpbs=(2, 4),
                    log=log)
    head = AT.tune(ix, tune_q, tune_gt, K=K, target=TUNE_TARGET, storages=(N.STORE_BF16,), Ms=Ms, wpbs=(2, 4),
                   learned_model=model, learned_opts=learned_opts if model is not None else (), log=log)
    tm["autotune_s"] = round(time.time() - t0, 1)
    if plain.kernel_ms < head.kernel_ms:
        head = plain
    if head.learned is not None:
        LE.attach(ix, model, **head.learned)
    log(f"plain fp32 L={plain.L} M={plain.M} {plain.kernel_ms:.3f} ms; head storage={head.storage} L={head.L} "
        f"M={head.M} learned={head.learned} {head.kernel_ms:.3f} ms")

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    sampler = ClockSampler(0)

    def timed(c):
        kw = c.search_kwargs()
        for _ in range(args.warmup):
            ix.search(K=K, **kw)
        torch.cuda.synchronize()
        kms, tot_, ids_ = 0.0, {"n_dist": 0, "n_edges": 0}, None
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ids_, st = ix.search(K=K, **kw)
            kms += st["kernel_ms"]
            for k_ in tot_:
                tot_[k_] += st[k_]
        torch.cuda.synchronize()
        return kms, tot_, ids_

    sampler.start()
    kernel_ms, tot, last_ids = timed(head)
    rec = recall(last_ids, gts, 100, 100)
    if head is plain:
        p_ms, p_tot, p_ids = kernel_ms, tot, last_ids
    else:
        p_ms, p_tot, p_ids = timed(plain)
    p_rec = recall(p_ids, gts, 100, 100)
    # End to end through the host-pointer call, pinned queries and ids.
    kw = head.search_kwargs()
    q_pin = torch.from_numpy(qs).pin_memory().numpy()
    out_pin = torch.empty((nq, K), dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    for _ in range(args.warmup):
        ix.search(q_pin, K=K, out=out_pin, **kw)
    e2e_s = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ix.search(q_pin, K=K, out=out_pin, **kw)
        e2e_s += time.perf_counter() - t0
    clocks = sampler.stop()

    # Uneven batches through the asynchronous device-pointer entry point with
    # the CUDA-graph-captured launch, back to back on one stream, at the
    # head's configuration and at L = 200 and 400 (recall of each L on the
    # evaluation queries).
    pool = torch.from_numpy(workloads.vectors(spec, 65_536, spec["query_seed"] + 7)).cuda()
    stream = torch.cuda.Stream()
    batches = {}
    for Lb in sorted({head.L, 200, 400}):
        # warps per query chosen by the library from the batch size
        kwb = dict(kw, L=Lb, flags=kw["flags"] | N.FLAG_CUDA_GRAPH, warps_per_query=0, warps_per_block=0,
                   blocks_per_sm=0)
        ids_b, _ = ix.search(K=K, **dict(kw, L=Lb))
        row = {"recall100": round(recall(ids_b, gts, 100, 100), 5)}
        for B in (1, 16, 256, 4096, 65_536):
            nb = max(2, min(200, 131_072 // B))
            outb = torch.empty((B, K), dtype=torch.int32, device="cuda")
            for i in range(2):
                s0 = (i * B) % (65_536 - B + 1)
                ix.search_device(pool[s0:s0 + B], outb, K=K, stream=stream, **kwb)
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for i in range(nb):
                s0 = (i * B) % (65_536 - B + 1)
                ix.search_device(pool[s0:s0 + B], outb, K=K, stream=stream, **kwb)
            e1.record(stream)
            stream.synchronize()
            ms = e0.elapsed_time(e1)
            row[str(B)] = round(nb * B / (ms / 1e3), 1)
        batches[f"L{Lb}"] = row
    log(f"batches: {batches}")

    steps = args.steps
    s_el = {N.STORE_FP32: 4, N.STORE_BF16: 2, N.STORE_FP8: 1}[head.storage]
    alg_bytes = (tot["n_dist"] * (s_el * d + 4) + 4 * tot["n_edges"]) / steps + nq * (4 * d + 4 * K)
    if head.storage != N.STORE_FP32:
        alg_bytes += nq * head.L * (4 * d + 4)
    achieved = alg_bytes / (kernel_ms / steps / 1e3) / 1e9
    p_alg = (p_tot["n_dist"] * (4 * d + 4) + 4 * p_tot["n_edges"]) / steps + nq * (4 * d + 4 * K)
    peak, peak_kind = measured_peak_hbm()
    names = {N.STORE_FP32: "fp32", N.STORE_BF16: "bf16", N.STORE_FP8: "fp8"}
    why = ("not run at this size: the reference's loaders build the whole index in host memory "
           "(load_nsg_graph interleaves ~600 B rows: ~60 GB, next to the 38 GB base), and its "
           "all-pairs tools cannot build this graph")
    line = {
        "metric": metric_for(spec), "value": round(nq * steps / (kernel_ms / 1e3), 1), "unit": UNIT, "n_gpus": 1,
        "steps": steps, "warmup": args.warmup, "ms_per_step": round(kernel_ms / steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": names[head.storage],
        "data": "synthetic",
        "config": {"workload": "batched search, " + workloads.describe(spec) + " (per GPU), in memory",
                   "graph": dict(ginfo, rule="exact 64-NN within each k-means cell and its 3 nearest cells, "
                                            "MRNG prune to R=48, reverse edges up to R, medoid entry, "
                                            "reachability repair"),
                   "L": head.L, "M": head.M, "warps_per_block": head.warps_per_block,
                   "storage": names[head.storage], "accumulate": "f32",
                   "rerank": "exact f32 of the final L" if head.storage != N.STORE_FP32 else None,
                   "learned": head.learned, "recall100": round(rec, 5),
                   "operating_point": "autotuned on 10k held-out queries",
                   "l2": "inputs > L2 and a 256 MB L2 flush before each step", "build_s": tm},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None, "peak_source": peak_kind},
        "e2e": {"value": round(nq * steps / e2e_s, 1), "unit": UNIT, "h2d_bytes_per_step": nq * d * 4,
                "d2h_bytes_per_step": nq * K * 4 + nq * 16 + 4},
        "gpu_launches": steps,
        "plain_fp32": {"value": round(nq * steps / (p_ms / 1e3), 1), "L": plain.L, "M": plain.M,
                       "recall100": round(p_rec, 5),
                       "roofline_frac": round(p_alg / (p_ms / steps / 1e3) / 1e9 / peak, 4)},
        "uneven_batches_qps": batches,
        "parity": {"unavailable": why},
        "clocks": clocks,
        "cpu_baseline": {"unavailable": why},
    }
    print(json.dumps(line), flush=True)
    ix.close()


def cpu_baseline(paths, L, nq_total, log):
    """The reference's PSS_v5 on every host core, on a bounded query sample
    (about 10-20 s of CPU work per mode), at the L of the GPU's plain operating
    point: the intra-query OpenMP search (X in {1, 4}) and the inter-query mode;
    `value` is the fastest."""
    try:
        T = nproc()
        modes = []
        for name, binary, X, inner in REF_MODES:
            try:
                probe = run_reference_pss(paths, min(300, nq_total), L, T, X=X, binary=binary, inner=inner)
                per_q = probe["runtime_s"] / probe["nq"]
                sample = int(max(200, min(nq_total, 10.0 / max(per_q, 1e-9))))
                r = run_reference_pss(paths, sample, L, T, X=X, binary=binary, inner=inner)
                modes.append({"mode": name, "X": X, "threads": r["threads"], "queries": r["nq"],
                              "qps": round(r["qps"], 1), "recall100": round(r["recall100"], 4)})
                log(f"cpu baseline: {name} T={T} X={X} L={L}: {r}")
            except Exception as e:  # one mode missing must not hide the others
                log(f"cpu baseline mode {name} unavailable: {e}")
        if not modes:
            return None
        best = max(modes, key=lambda m: m["qps"])
        return {"value": best["qps"], "unit": UNIT, "cores": T, "kind": "reference",
                "sample": f"{best['queries']} of the queries, {best['mode']} (L={L}, X={best['X']}, "
                          f"{best['threads']} threads), recall@100 {best['recall100']:.4f}, {cpu_model()}; "
                          f"all modes timed: " + "; ".join(f"{m['mode']} X={m['X']}: {m['qps']} QPS"
                                                             for m in modes),
                "modes": modes}
    except Exception as e:  # the baseline is informative; never fail the bench on it
        log(f"cpu baseline unavailable: {e}")
        return None


# ---------------------------------------------------------------------------
def bench_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    from parallel_anns_b200 import workloads
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_pss")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference binaries were not built (oracle/_ref/ref_pss missing)"}))
        return
    spec = workloads.SPECS[args.workload](**({"n": args.n} if args.n else {}), nq=args.nq)
    args.n = spec["n"]
    # Inputs: the cached files if present, else built on the host (no GPU
    # library in this process).
    if workloads.cached(spec):
        W = workloads.load(spec)
    elif spec.get("kind") == "uint8":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the integer-valued workload's inputs are built on the GPU only (no cluster "
                          "structure for the host builder); run the GPU arm first"}))
        return
    else:
        W = host_workload(spec, log)
    T = nproc()
    # The reference's own operating point: smallest swept L with recall@100 >= 0.95
    # on a sample, measured by the reference itself.
    L = args.L
    if not L:
        for Lc in L_SWEEP:
            r = run_reference_pss(W["paths"], min(1000, args.nq), Lc, T)
            if r["recall100"] >= RECALL_TARGET:
                L = Lc
                break
        L = L or L_SWEEP[-1]
    # The faster of the reference's CPU modes at that L (intra-query PSS_v5 or
    # its inter-query multi_queries_LG form), each on all host cores.
    best = None
    for name, binary, X, inner in REF_MODES:
        if binary != "ref_pss" and not os.path.exists(os.path.join(ROOT, "oracle", "_ref", binary)):
            continue
        pr = run_reference_pss(W["paths"], min(500, args.nq), L, T, X=X, binary=binary, inner=inner)
        if best is None or pr["qps"] > best[0]["qps"]:
            best = (pr, name, binary, X, inner)
    probe, mode_name, binary, X, inner = best
    per_q = probe["runtime_s"] / probe["nq"]
    budget_s = 150.0 / max(1, args.steps + args.warmup)
    sample = int(max(100, min(args.nq, budget_s / max(per_q, 1e-9))))
    r = run_reference_pss(W["paths"], sample, L, T, X=X, reps=args.warmup + args.steps, binary=binary,
                          inner=inner)
    times = r["rep_times"][args.warmup:]
    value = sample * len(times) / sum(times)
    line = {"metric": metric_for(spec), "value": round(value, 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "batched search, " + workloads.describe(spec),
                       "n": args.n, "d": spec["d"], "K": 100, "L": L, "T": T, "X": X, "mode": mode_name,
                       "recall100": r["recall100"], "queries_per_step": sample},
            "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": T, "kind": "reference",
                             "sample": f"{sample} queries per step, {mode_name}, L_master=L_local={L}, "
                                       f"X={X}, T={T}, {cpu_model()}"},
            "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=None, help="base size (default: the workload's)")
    ap.add_argument("--nq", type=int, default=10_000, help="queries per GPU")
    ap.add_argument("--L", type=int, default=0, help="fix L (default: recall-driven sweep)")
    ap.add_argument("--M", type=int, default=0, help="fix M (default: sweep)")
    ap.add_argument("--storage", type=int, default=None, choices=[0, 1, 2],
                    help="fix the storage (0 fp32, 1 bf16, 2 fp8; default: sweep)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="leave the learned entry network out")
    ap.add_argument("--no-parity", action="store_true", help="skip the id check against the reference")
    ap.add_argument("--wpb", type=int, default=2, help="warps per block with a fixed --L and --M")
    ap.add_argument("--entries", default=None,
                    help="with a fixed --L and --M: learned entries E:L_init[:min_conf] (the network is trained first)")
    ap.add_argument("--workload", default="mixture_1m_d96",
                    choices=["mixture_1m_d96", "u8_1m_d128", "mixture_10m_d96", "mixture_100m_d96"],
                    help="mixture_1m_d96: the batched-FP32 config (default); u8_1m_d128: the "
                         "reduced-precision config's integer-valued d = 128 variant (R = 64); mixture_10m_d96: "
                         "the learned-entry config's 10M base")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        bench_reference(args)
    else:
        bench_ours(args)


if __name__ == "__main__":
    main()
