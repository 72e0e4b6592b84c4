"""The learned entry / L-budget part on the GPU, through the C ABI.

* The network's GPU forward pass, loss and gradient (the kernels training
  runs) agree with the float64 CPU oracle (tests/test_learned_oracle.py pins
  that oracle) to float32 accumulation error.
* Training lowers the loss; k-means returns distinct representatives that
  lie in their own cells.
* The learned search is exact given its decisions: the batched inference's per-query
  decision (fallback, queue length, entry vertices) matches the oracle's, and
  the ids equal the oracle's top-M search from those entries; with a network
  that is never confident, every query runs the plain search, id for id.
* The trained network needs fewer distance computations than the plain
  method for the same recall.
"""
import numpy as np
import pytest

import mlp_oracle as MO
import oracle as O

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("d,R,B,T", [(96, 1024, 64, 10), (24, 256, 37, 3)])
def test_loss_grad_matches_oracle(d, R, B, T):
    from parallel_anns_b200 import learned as LE
    rng = np.random.default_rng(d + R)
    X = rng.standard_normal((B, d)).astype(np.float32) * 0.3
    cells = rng.integers(0, R, (B, T)).astype(np.uint16)
    y = rng.normal(5.5, 0.4, B).astype(np.float32)
    p = LE.init_params(d, R, seed=5, y_mean=5.0)
    p += rng.normal(0, 0.01, p.size).astype(np.float32)  # non-zero biases
    loss, g = LE.loss_grad(p, X, cells, y, R, lam=0.8)
    rl, rg = MO.loss_grad(p, X, cells, y, d, R, 0.8, bf16=True)
    assert abs(loss - rl) <= 1e-5 * abs(rl)
    parts_g, parts_r = MO.unpack(g, d, R), MO.unpack(rg, d, R)
    for name, a, b in zip(("W1", "b1", "W2", "b2", "W3", "b3"), parts_g, parts_r):
        assert rel_err(a, b) < 2e-4, (name, rel_err(a, b))
    Z = LE.forward(p, X, R)
    _, _, rZ, _ = MO.forward(p, X, d, R, True)
    assert rel_err(Z, rZ) < 1e-5


def test_training_lowers_loss_and_learns_cells():
    """A learnable task: the label of x is the nearest of R random centres."""
    from parallel_anns_b200 import learned as LE
    d, R, n = 32, 256, 20000
    rng = np.random.default_rng(11)
    C = rng.standard_normal((R, d)).astype(np.float32)
    X = (C[rng.integers(0, R, n)] + 0.3 * rng.standard_normal((n, d))).astype(np.float32)
    lab = np.argmin(((X[:, None, :] - C[None]) ** 2).sum(-1), 1)
    cells = lab[:, None].astype(np.uint16)
    y = (4.0 + 0.5 * X[:, 0]).astype(np.float32)
    p, losses = LE.train(X, cells, y, R, epochs=6, batch=512, lr=2e-3)
    assert losses[-1] < 0.5 * losses[0], losses
    Z = LE.forward(p, X[:2000], R)
    acc = np.mean(Z[:, :R].argmax(1) == lab[:2000])
    assert acc > 0.8, acc
    assert np.mean(np.abs(Z[:, R] - y[:2000])) < 0.2


@pytest.fixture(scope="module")
def small():
    from parallel_anns_b200 import datasets as ds
    from parallel_anns_b200.searching import Index
    base = ds.gaussian_mixture(30000, 96, seed=501, means_seed=501)
    q = ds.gaussian_mixture(300, 96, seed=502, means_seed=501)
    from parallel_anns_b200.graph import build_nsg
    g = build_nsg(base, R=50, knn_k=64)  # the library's construction: the same graph in every process
    ix = Index(0)
    ix.set_base(base)
    ix.set_graph(g)
    ix.set_queries(q)
    yield ix, base, q, g
    ix.close()


def test_kmeans_representatives(small):
    from parallel_anns_b200 import learned as LE
    ix, base, q, g = small
    reps, assign = LE.kmeans(ix, 256, 10, seed=3)
    assert len(set(reps.tolist())) == 256
    counts = np.bincount(assign, minlength=256)
    nonempty = counts > 0
    assert nonempty.sum() > 200
    assert np.all(assign[reps[nonempty]] == np.nonzero(nonempty)[0])
    reps2, assign2 = LE.kmeans(ix, 256, 10, seed=3)
    assert np.array_equal(reps, reps2) and np.array_equal(assign, assign2)  # deterministic


def check_learned_search(ix, base, q, g, model, K, L, M, lp):
    from parallel_anns_b200 import learned as LE
    from parallel_anns_b200 import native as N
    LE.attach(ix, model, **lp)
    ids, st = ix.search(K=K, L=L, mode=N.MODE_TOP_M if M > 1 else N.MODE_NSG_SEQ, M=M, flags=N.FLAG_LEARNED)
    Lq, fb, entries = LE.record(ix, q.shape[0])
    dec = MO.decide(model.params, q, 96, model.R, model.reps, K=K, L=L, **{
        "E": lp["E"], "L_init": lp.get("L_init", 1 << 30), "L_min": lp.get("L_min", 0),
        "use_L": int(lp.get("use_L", True)), "L_scale": lp.get("L_scale", 1.0),
        "L_exp": lp.get("L_exp", 1.0), "min_conf": lp.get("min_conf", 0.0)})
    # decisions agree with the oracle (up to float32 near-ties)
    agree = 0
    for i, (ofb, oLq, oent, _, conf, r, lg) in enumerate(dec):
        same = ofb == fb[i] and oLq == Lq[i] and list(entries[i]) == oent
        agree += same
    assert agree >= 0.97 * len(dec), agree
    # ids equal the oracle search started from the GPU's own decisions
    G = O.Graph.from_nsg(g)
    plain = ix.prepare_init_ids(L)
    lists = []
    for i in range(q.shape[0]):
        if fb[i]:
            lists.append(plain[:L])
        else:
            e = list(entries[i])
            n_plain = Lq[i] - len(e)
            if e:
                n_plain = min(n_plain, lp.get("L_init", 1 << 30))
            lists.append(np.array(e + list(plain[:n_plain]), dtype=np.uint32))
    ref, nd = O.search_top_m_lists(base, G, q, K, Lq, M, lists)
    bad = np.nonzero((ids != ref).any(1))[0]
    assert bad.size == 0, bad[:10]
    assert st["n_dist"] == nd
    # several warps per query from the same decisions: the same ids and counts
    for wq in (2, 4):
        ids_w, st_w = ix.search(K=K, L=L, mode=N.MODE_TOP_M if M > 1 else N.MODE_NSG_SEQ, M=M, flags=N.FLAG_LEARNED,
                                warps_per_query=wq)
        assert np.array_equal(ids_w, ids) and st_w["n_dist"] == nd, wq
    return ids, Lq, fb


def test_learned_search_exact_given_decisions(small):
    from parallel_anns_b200 import learned as LE
    ix, base, q, g = small
    reps, _ = LE.kmeans(ix, 256, 5, seed=4)
    p = LE.init_params(96, 256, seed=9, y_mean=np.log(150.0))
    rng = np.random.default_rng(1)
    p[-257:] += rng.normal(0, 0.5, 257).astype(np.float32)  # spread logits and the L output
    model = LE.LearnedModel(96, 256, p, reps)
    for lp, M in ((dict(E=16, L_init=1 << 30, use_L=True, L_scale=1.0), 4),
                  (dict(E=8, L_init=24, use_L=True, L_scale=0.8, L_exp=0.6, L_min=64), 1),
                  (dict(E=40, L_init=0, use_L=False), 8)):
        check_learned_search(ix, base, q, g, model, 50, 200, M, lp)


def test_learned_search_exact_given_decisions_many_classes(small):
    """More entry classes than the batched inference keeps in registers
    (R = 2,048: the logits are read from its scratch)."""
    from parallel_anns_b200 import learned as LE
    ix, base, q, g = small
    rng = np.random.default_rng(7)
    reps = rng.choice(base.shape[0], 2048, replace=False).astype(np.uint32)
    p = LE.init_params(96, 2048, seed=11, y_mean=np.log(150.0))
    p[-2049:] += rng.normal(0, 0.5, 2049).astype(np.float32)  # spread logits and the L output
    model = LE.LearnedModel(96, 2048, p, reps)
    check_learned_search(ix, base, q, g, model, 50, 200, 4, dict(E=16, L_init=8, use_L=True, L_scale=1.0))


def test_unconfident_network_runs_plain_search(small):
    from parallel_anns_b200 import learned as LE
    from parallel_anns_b200 import native as N
    ix, base, q, g = small
    reps = np.arange(256, dtype=np.uint32) * 7
    p = np.zeros(LE.param_count(96, 256), np.float32)  # equal logits: confidence 1/256
    LE.attach(ix, LE.LearnedModel(96, 256, p, reps), E=16, use_L=True, L_scale=0.1, min_conf=0.01)
    ids, st = ix.search(K=100, L=160, mode=N.MODE_TOP_M, M=4, flags=N.FLAG_LEARNED)
    ref, st0 = ix.search(K=100, L=160, mode=N.MODE_TOP_M, M=4)
    assert np.array_equal(ids, ref) and st["n_dist"] == st0["n_dist"]
    Lq, fb, entries = LE.record(ix, q.shape[0])
    assert fb.all() and (Lq == 160).all()


def test_trained_network_gains_over_plain(small):
    """Same recall target, fewer distance computations: the plain method's
    cheapest L reaching recall 0.95 against the exact neighbours, versus the
    learned search tuned on held-out queries (not the evaluated ones)."""
    from parallel_anns_b200 import datasets as ds
    from parallel_anns_b200 import learned as LE
    from parallel_anns_b200 import native as N
    from parallel_anns_b200.searching import ground_truth, recall
    ix, base, q, g = small
    train_q = ds.gaussian_mixture(20000, 96, seed=503, means_seed=501)
    tune_q = ds.gaussian_mixture(1000, 96, seed=504, means_seed=501)
    eval_q = ds.gaussian_mixture(1000, 96, seed=505, means_seed=501)
    model = LE.build_model(ix, train_q, R=256, K=100, M=4, L_ref=600, T=10, epochs=10, batch=512,
                           kmeans_iters=10, seed=2)
    gt_tune, _ = ground_truth(ix, tune_q, 100)
    gt_eval, _ = ground_truth(ix, eval_q, 100)

    def plain(qs, L):
        ids, st = ix.search(qs, K=100, L=L, mode=N.MODE_TOP_M, M=4)
        return ids, st["n_dist"]

    def learned(qs, L, scale):
        LE.attach(ix, model, E=16, L_init=16, use_L=True, L_scale=scale, L_min=100)
        ids, st = ix.search(qs, K=100, L=L, mode=N.MODE_TOP_M, M=4, flags=N.FLAG_LEARNED)
        return ids, st["n_dist"]

    Ls = [100, 120, 140, 160, 190, 220, 260, 300, 360, 420, 500]
    # plain: cheapest L reaching the target on the tuning queries
    Lp = next(L for L in Ls if recall(plain(tune_q, L)[0], gt_tune, L, 100) >= 0.95)
    # learned: cheapest scale reaching it on the tuning queries
    scales = [0.6, 0.7, 0.8, 0.9, 1.0, 1.15, 1.3, 1.5, 1.75, 2.0, 2.5, 3.0]
    sl = next(s for s in scales if recall(learned(tune_q, 500, s)[0], gt_tune, 100, 100) >= 0.95)
    ids_p, nd_p = plain(eval_q, Lp)
    ids_l, nd_l = learned(eval_q, 500, sl)
    rp = recall(ids_p, gt_eval, 100, 100)
    rl = recall(ids_l, gt_eval, 100, 100)
    print(f"plain L={Lp}: recall {rp:.4f} n_dist {nd_p}; learned scale {sl}: recall {rl:.4f} n_dist {nd_l} "
          f"({nd_p / nd_l:.2f}x fewer)")
    assert rl >= 0.95 - 0.005
    assert nd_l < 0.95 * nd_p
