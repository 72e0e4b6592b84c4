"""Multi-rank host logic of the replica layout, on CPU with gloo ranks
(world_size 2): query shards are disjoint and cover the set, the timed value is
the maximum over ranks, and the operating point chosen on rank 0 reaches every
rank."""
import os

import pytest
import torch.multiprocessing as mp


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from parallel_anns_b200.replicas import Ranks, env, shard
    r, w, lr = env()
    ranks = Ranks(w, device="cpu")
    sl = shard(r, 100)
    ranks.barrier()
    mx = ranks.max(1.5 + r)
    choice = ranks.broadcast_ints([7 + r, 400, 8], 0)
    # the bench's operating point (autotuner choice, a JSON object) from rank 0
    obj = ranks.broadcast_json({"head": {"storage": 2, "L": 384, "learned": None}, "rank": r} if r == 0 else None, 0)
    q.put((r, w, lr, sl.start, sl.stop, mx, choice, obj))
    dist.destroy_process_group()


def test_two_gloo_ranks():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, l0, a0, b0, m0, c0, o0), (r1, w1, l1, a1, b1, m1, c1, o1) = out
    assert (r0, r1, w0, w1) == (0, 1, 2, 2)
    assert (a0, b0, a1, b1) == (0, 100, 100, 200)
    assert m0 == m1 == 2.5
    assert c0 == c1 == [7, 400, 8]
    assert o0 == o1 == {"head": {"storage": 2, "L": 384, "learned": None}, "rank": 0}
