"""Host-side pieces of the benchmark: workload specs, metric names, and the
host-built inputs the reference arm uses (no GPU, no library)."""
import importlib.util
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_metric_names_follow_the_workload():
    from parallel_anns_b200 import workloads
    b = load_bench()
    assert b.metric_for(workloads.SPECS["mixture_1m_d96"]()) == b.METRIC
    assert "10M x 96d" in b.metric_for(workloads.SPECS["mixture_10m_d96"]())
    assert "1M x 128d" in b.metric_for(workloads.SPECS["u8_1m_d128"]())
    assert "100M x 96d" in b.metric_for(workloads.SPECS["mixture_100m_d96"]())


def test_large_workload_spec():
    """The 100M configuration: 4,096 mixture components, R = 48, 10,000 cells
    with 3 probed neighbours, reverse edges, one learned class per component,
    held in memory; smaller bases scale the cell count (1 per 1,000 vectors)."""
    from parallel_anns_b200 import workloads
    s = workloads.SPECS["mixture_100m_d96"]()
    assert (s["n"], s["d"], s["components"], s["R"], s["knn_k"]) == (100_000_000, 96, 4096, 48, 64)
    assert (s["cells"], s["probe"], s["reverse"], s["reps"], s["large"]) == (10_000, 3, True, 4096, True)
    assert workloads.SPECS["mixture_100m_d96"](n=2_000_000)["cells"] == 2000
    b = load_bench()
    assert b.TUNE_TARGET > b.RECALL_TARGET


def test_host_workload_matches_store_and_load(tmp_path, monkeypatch):
    """The reference arm's host build writes the reference's formats and a
    meta record that the GPU arm's cache lookup accepts."""
    from parallel_anns_b200 import workloads
    monkeypatch.setattr(workloads, "CACHE", str(tmp_path))
    b = load_bench()
    spec = workloads.SPECS["mixture_1m_d96"](n=5000, nq=50)
    assert not workloads.cached(spec)
    W = b.host_workload(spec, log=None)
    assert workloads.cached(spec)
    L = workloads.load(spec)
    assert L["meta"]["built_by"] == b.HOST_BUILT
    assert np.array_equal(L["base"], W["base"]) and np.array_equal(L["gt"], W["gt"])
    assert L["graph"].entry == W["graph"].entry and np.array_equal(L["graph"].nbrs, W["graph"].nbrs)
