"""The CPU oracle of the entry / L-budget network is itself pinned before it
checks the GPU: its analytic gradient matches central differences of its own
loss, its BF16 rounding matches known bit patterns (round to nearest, ties to
even), and the per-query decision follows its stated rules."""
import numpy as np
import pytest

import mlp_oracle as MO


def small_batch(d=16, R=256, B=6, T=5, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((B, d)).astype(np.float32)
    cells = rng.integers(0, R, (B, T)).astype(np.uint16)
    y = rng.normal(5.0, 0.5, B).astype(np.float32)
    p = MO.init_params(d, R, seed)
    p[MO.param_count(d, R) - 1] = 5.0  # L output bias near the targets
    return p, X, cells, y


def test_param_layout_count():
    assert MO.param_count(96, 1024) == 96 * 256 + 256 + 256 * 256 + 256 + 256 * 1025 + 1025
    p = np.arange(MO.param_count(8, 256), dtype=np.float64)
    parts = MO.unpack(p, 8, 256)
    assert [x.shape for x in parts] == [(8, 256), (256,), (256, 256), (256,), (256, 257), (257,)]
    assert np.array_equal(MO.pack(parts), p)


def test_analytic_gradient_matches_central_differences():
    d, R = 16, 256
    p, X, cells, y = small_batch(d, R)
    lam = 0.7
    _, g = MO.loss_grad(p, X, cells, y, d, R, lam, bf16=False)
    rng = np.random.default_rng(3)
    n = p.size
    # indices in every tensor, including the L output column and bias
    lay = np.cumsum([0, d * 256, 256, 256 * 256, 256, 256 * (R + 1), R + 1])
    idx = np.concatenate([rng.integers(lay[i], lay[i + 1], 12) for i in range(6)] +
                         [np.arange(lay[4] + R, lay[5], R + 1)[:8], [n - 1]])
    num = MO.numeric_grad(p, X, cells, y, d, R, lam, idx)
    ana = g[idx]
    assert np.allclose(ana, num, rtol=1e-4, atol=1e-7), np.max(np.abs(ana - num))


def test_bf16_round_to_nearest_even():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.0e-39], dtype=np.float32)
    got = MO.bf16_round(vals)
    # 1 + 2^-8 is half-way between 1 and 1 + 2^-7: ties to even -> 1.0;
    # 1 + 3*2^-8 is half-way between 1 + 2^-7 and 1 + 2^-6: ties to even -> 1 + 2^-6.
    want = np.array([1.0, 1.0, 1.0 + 2 ** -6, 1.0, -2.5, np.float32(3.0e-39)], dtype=np.float64)
    want[5] = MO.bf16_round(np.array([3.0e-39], np.float32))[0]
    assert np.array_equal(got[:5], want[:5])
    u = np.array([got[5]], np.float32).view(np.uint32)[0]
    assert u & 0xFFFF == 0


def test_decision_rules():
    d, R = 8, 256
    p = np.zeros(MO.param_count(d, R), np.float32)
    lay = np.cumsum([0, d * 256, 256, 256 * 256, 256, 256 * (R + 1), R + 1])
    X = np.zeros((2, d), np.float32)
    reps = np.arange(1000, 1000 + R, dtype=np.uint32)
    # equal logits: confidence 1/R -> fallback with any min_conf above it
    dec = MO.decide(p, X, d, R, reps, E=8, L_init=5, L_min=0, use_L=1, L_scale=1.0, min_conf=0.01,
                    K=10, L=300)
    assert all(x[0] and x[1] == 300 and x[2] == [] and x[3] == 300 for x in dec)
    # logits b3: cell 7 largest, then 3, 200 (ties -> lower index); L output ln(49.7)
    b3 = p[lay[5]:lay[6]]
    b3[7], b3[3], b3[200], b3[9] = 5.0, 4.0, 4.0, 3.0
    b3[R] = np.log(49.7)  # 2 * 49.7 = 99.4 -> L_q = 100
    dec = MO.decide(p, X, d, R, reps, E=3, L_init=5, L_min=0, use_L=1, L_scale=2.0, min_conf=0.0,
                    K=10, L=300)
    fb, Lq, ent, n_plain = dec[0][:4]
    assert not fb and Lq == 100 and ent == [1007, 1003, 1200] and n_plain == 5
    dec = MO.decide(p, X, d, R, reps, E=3, L_init=1000, L_min=120, use_L=1, L_scale=2.0, min_conf=0.0,
                    K=10, L=300)
    assert dec[0][1] == 120 and dec[0][3] == 117
