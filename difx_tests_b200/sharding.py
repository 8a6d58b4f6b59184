"""Work split across GPUs (one process per GPU over torch.distributed) and the
host-side reductions that go with it.

The correlation of one subintegration shards without a data-path exchange:
subbands and whole subintegrations are independent, and a subintegration's FFT
range splits into time shards whose accumulators add -- the reference's
split/merge (main.c:398-433 runs `split` partial accumulations, kernel.c:856-878
sums them).  So the multi-GPU forms are

* replicas: every rank correlates its own subintegration (weak scaling);
* subband shards: rank r correlates subbands shard(nsb, world, r); the
  visibilities are gathered once at the end;
* time shards: rank r correlates FFTs shard(numffts, world, r) of every subband;
  one sum of the visibilities and counts over ranks (NCCL all-reduce on GPUs)
  merges them, like the reference's `merge`.

Timings are the maximum over ranks of each rank's device time.
"""
from __future__ import annotations

import numpy as np


def shard(n: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced split of n items: (first, count) of `rank` (the first
    n % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("bad shard request")
    base, extra = divmod(n, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar (a device time) over the process group."""
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def merge_time_shards(vis: np.ndarray, counts: np.ndarray, device=None):
    """Sum of every rank's accumulated (un-normalised) visibilities and baseline
    counts: the time shards of one subintegration merged (kernel.c:856-878).
    Normalise after merging."""
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return vis, counts
    import torch
    v = torch.from_numpy(np.ascontiguousarray(vis).view(np.float32).copy()).to(device)
    c = torch.from_numpy(np.ascontiguousarray(counts, dtype=np.int64).copy()).to(device)
    dist.all_reduce(v)
    dist.all_reduce(c)
    return (v.cpu().numpy().view(np.complex64).reshape(vis.shape),
            c.cpu().numpy().astype(counts.dtype))


def gather_subbands(vis_local: np.ndarray, nsb_total: int, device=None) -> np.ndarray:
    """Visibilities [nsb_local][...] of every rank's subband shard (shard(nsb_total,
    world, rank)), concatenated in subband order on every rank."""
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return vis_local
    import torch
    world = dist.get_world_size()
    per_sb = vis_local.shape[1:]
    nmax = -(-nsb_total // world)
    buf = np.zeros((nmax,) + per_sb, np.complex64)
    buf[: vis_local.shape[0]] = vis_local
    t = torch.from_numpy(buf.view(np.float32).copy()).to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    out = []
    for r, p in enumerate(parts):
        _, n = shard(nsb_total, world, r)
        out.append(p.cpu().numpy().view(np.complex64).reshape((nmax,) + per_sb)[:n])
    return np.concatenate(out, axis=0)
