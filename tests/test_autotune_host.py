"""Host logic of the autotuner, without a GPU: a fake index whose recall grows
with L and whose time depends on the block shape. The tuner must find the
smallest grid L meeting the target (binary search), time only shapes that fit,
return the fastest, and cache the choice per shape."""
import json
import os
import tempfile

import numpy as np
import pytest

from parallel_anns_b200 import autotune as AT
from parallel_anns_b200 import native as N


class FakeIndex:
    n, d = 1000, 16

    def __init__(self):
        self.calls = []

    def search(self, queries, K=100, L=100, M=1, warps_per_block=0, blocks_per_sm=0, warps_per_query=1,
               storage=0, flags=0, mode=0):
        self.calls.append((L, M, warps_per_block, blocks_per_sm, warps_per_query))
        if warps_per_block == 4 and L >= 448:
            raise N.PannsError(-1, "search: the queue does not fit in shared memory")
        nq = queries.shape[0]
        # recall: the fraction of true ids returned grows with L (more for larger M)
        hits = min(100, int(60 + L / 10 + 4 * M))
        ids = np.tile(np.arange(100, dtype=np.uint32), (nq, 1))
        ids[:, hits:] += 5000
        ms = L / 100.0 * (1.0 + 0.1 * warps_per_block) / M ** 0.5 + 0.05 * blocks_per_sm
        return ids, {"kernel_ms": ms}


def test_autotuner_smallest_L_fastest_shape_and_cache():
    ix = FakeIndex()
    q = np.zeros((10, 16), np.float32)
    gt = np.tile(np.arange(100, dtype=np.uint32), (10, 1))
    grid = (100, 200, 300, 400, 448, 512)
    with tempfile.TemporaryDirectory() as t:
        cache = os.path.join(t, "tune.json")
        c = AT.tune(ix, q, gt, K=100, target=0.95, Ms=(1, 4), wpbs=(2, 4), bpss=(0, 5), L_grid=grid,
                    reps=1, cache=cache)
        # M = 1 reaches 95 hits at L = 350 -> 400; M = 4 at L = 190 -> 200
        assert (c.M, c.L) == (4, 200)
        assert c.warps_per_block == 2 and c.blocks_per_sm == 0  # the cheaper shape in the fake
        rows = [r for r in c.table if r.get("L")]
        assert {(r["M"], r["L"]) for r in rows} == {(1, 400), (4, 200)}
        assert all(r["recall"] >= 0.95 for r in rows)
        saved = json.load(open(cache))
        assert len(saved) == 1
        n_calls = len(ix.calls)
        c2 = AT.tune(ix, q, gt, K=100, target=0.95, Ms=(1, 4), wpbs=(2, 4), bpss=(0, 5), L_grid=grid,
                     reps=1, cache=cache)
        assert len(ix.calls) == n_calls and (c2.M, c2.L, c2.warps_per_block) == (4, 200, 2)


def test_autotuner_skips_shapes_that_do_not_fit_and_reports_unreachable():
    ix = FakeIndex()
    q = np.zeros((4, 16), np.float32)
    gt = np.tile(np.arange(100, dtype=np.uint32), (4, 1))
    c = AT.tune(ix, q, gt, K=100, target=0.99, Ms=(1,), wpbs=(2, 4), bpss=(0,), L_grid=(100, 448, 512),
                reps=1)
    assert c.L == 448 and c.warps_per_block == 2  # 4 warps per block do not fit L >= 448
    with pytest.raises(RuntimeError):
        AT.tune(ix, q, gt, K=100, target=1.01, Ms=(1,), wpbs=(2,), bpss=(0,), L_grid=(100, 200), reps=1)
