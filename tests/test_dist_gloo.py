"""Multi-rank host logic on CPU with the gloo backend (world size 2 and 3):
frame sharding covers every frame exactly once and the gather reassembles
the stack in order on every rank."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from ncs_b200.dist import shard_and_gather
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        T, H, W = 7, 5, 4
        images = torch.arange(T * H * W, dtype=torch.float32).reshape(T, H, W)
        seen = []

        def solve(x):
            seen.append(x.shape[0])
            return x * 2.0 + 1.0

        out = shard_and_gather(images, solve)
        ok = torch.equal(out, images * 2.0 + 1.0)
        # max-over-ranks timing as bench.py does
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        q.put((rank, ok, sum(seen), float(t.item())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_shard_and_gather_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok for _, ok, _, _ in res)
    assert sum(n for _, _, n, _ in res) == 7          # every frame solved exactly once
    assert all(t == float(world) for _, _, _, t in res)


def test_frame_range():
    from ncs_b200.dist import frame_range
    for T in range(0, 20):
        for world in range(1, 9):
            spans = [frame_range(T, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == T
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c and b >= a
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def _bench_worker(rank, world, port, q):
    import datetime
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        # per-rank times and pixel counts: the job's time is the slowest
        # rank's, its pixels the sum over ranks
        q.put((rank, bench.max_over_ranks(10.0 + rank, world),
               bench.sum_over_ranks(100.0 * (rank + 1), world)))
    finally:
        dist.destroy_process_group()


def test_bench_rank_reductions_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(mx == 11.0 and sm == 300.0 for _, mx, sm in res)
