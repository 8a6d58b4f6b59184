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


def _collective_device(device):
    """Where collective buffers live: the GPU under NCCL, host memory under gloo."""
    dist = _dist()
    if dist is not None and dist.get_backend() == "nccl":
        return device
    return "cpu"


def shard_config(fx, cfg, mode: str, world: int, rank: int):
    """This rank's correlator configuration and where its input starts.

    mode "time": every subband, FFTs shard(numffts, world, rank) -> (cfg, first_fft, nfft, first_sb=0)
    mode "subband": subbands shard(nsubband, world, rank), every FFT; the LO of the rank's first
    subband becomes its subband 0 -> (cfg_r, 0, numffts, first_sb)."""
    import copy
    if mode == "time":
        f0, n = shard(cfg.numffts, world, rank)
        return cfg, f0, n, 0
    if mode == "subband":
        s0, ns = shard(cfg.nsubband, world, rank)
        c = copy.copy(cfg)
        c.nsubband = max(ns, 1)
        c.lo = cfg.lo + cfg.sb_spacing * s0
        return c, 0, cfg.numffts, s0
    raise ValueError(f"unknown shard mode {mode}")


def correlate_shard(fx, corr, mode: str, d_data: int, pitch: int, delays, offs, first_fft: int, nfft: int,
                    first_sb: int, nsb_total: int, device, normalize=False):
    """One subintegration split over the process group, correlated through the library on every
    rank and merged on the device (under NCCL):

    * "time": this rank's FFT range of every subband, then one all-reduce sum of the un-normalised
      visibilities and of the counts (the reference's merge, kernel.c:856-878), normalised after;
    * "subband": this rank's subbands (corr configured by shard_config), then one all-gather.

    d_data: device rows [nsubband][nant][pitch] of the whole subintegration.  Returns (vis torch
    tensor float32 [2 * vis_count of the whole problem] on `device`, counts int64 tensor)."""
    import torch
    dist = _dist()
    world = dist.get_world_size() if dist is not None else 1
    cdev = _collective_device(device)
    corr.reset()
    nrows = corr.nant * (first_sb if mode == "subband" else 0)
    if nfft > 0 and (mode == "time" or shard(nsb_total, world, dist.get_rank() if dist else 0)[1] > 0):
        corr.process_device(d_data + nrows * pitch, pitch, delays, offs, first_fft, nfft)
    vis = torch.empty(2 * corr.vis_count, dtype=torch.float32, device=device)
    counts = torch.from_numpy(corr.visibilities_device(vis.data_ptr(), normalize=False).astype(np.int64))
    if mode == "time":
        if world > 1:
            v, c = vis.to(cdev), counts.to(cdev)
            dist.all_reduce(v)
            dist.all_reduce(c)
            vis, counts = v.to(device), c.cpu()
        if normalize:
            per_bl = vis.view(corr.nsb, corr.nbl + corr.nant, -1)
            cd = counts.to(device=device, dtype=torch.float32).clamp(min=1.0)
            per_bl /= cd[None, :, None]
        return vis, counts
    # subband shards: gather in subband order (a rank without subbands contributes zeros)
    per_sb = 2 * corr.vis_count // corr.nsb
    nmax = -(-nsb_total // world)
    buf = torch.zeros(nmax * per_sb, dtype=torch.float32, device=cdev)
    _, ns = shard(nsb_total, world, dist.get_rank() if dist else 0)
    buf[: ns * per_sb] = vis[: ns * per_sb].to(cdev)
    if normalize and ns:
        per_bl = buf[: ns * per_sb].view(ns, corr.nbl + corr.nant, -1)
        per_bl /= counts.to(device=cdev, dtype=torch.float32).clamp(min=1.0)[None, :, None]
    if world == 1:
        return buf.to(device), counts
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = torch.cat([p[: shard(nsb_total, world, r)[1] * per_sb] for r, p in enumerate(parts)])
    return out.to(device), counts
