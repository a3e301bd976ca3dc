"""Multi-GPU: the stack shards by frame with no exchange step.

Each rank solves a contiguous range of frames on its own GPU; the optional
gather at the end is one all_gather (NCCL over NVLink between GPUs, gloo on
CPU).  Nothing crosses devices inside the solve.
"""
import torch


def frame_range(n_frames, world, rank):
    """Contiguous, balanced [start, stop) of frames for `rank` (the first
    n_frames % world ranks take one extra frame)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n_frames, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard_and_gather(images, solve, group=None, gather=True):
    """Run `solve` on this rank's frames of `images` [T, ...] and, if `gather`,
    all_gather the results so every rank returns the full [T, ...] result.

    `solve` maps a [t, ...] tensor to a same-shaped tensor on the same device
    (e.g. ``lambda x: solver.reduce_noise(x, gamma)``).  With one rank this is
    just ``solve(images)``."""
    import torch.distributed as dist
    if group is None and not dist.is_initialized():
        return solve(images)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    T = images.shape[0]
    a, b = frame_range(T, world, rank)
    mine = solve(images[a:b]) if b > a else images[a:a]
    if not gather:
        return mine
    cap = -(-T // world)
    padded = torch.zeros((cap,) + tuple(images.shape[1:]), dtype=mine.dtype, device=mine.device)
    padded[: b - a] = mine
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    out = []
    for r in range(world):
        ra, rb = frame_range(T, world, r)
        out.append(parts[r][: rb - ra])
    return torch.cat(out, dim=0)
