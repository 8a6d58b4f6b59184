"""Multi-GPU host logic on CPU: two `gloo` ranks split a subintegration into
time shards (merged by one sum, the reference's split/merge) and into subband
shards (gathered), and reduce a per-rank time to its maximum.  The oracle stands
in for each rank's device correlation; the merged results must equal the
single-rank correlation of the whole subintegration."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from difx_tests_b200 import sharding


def test_shard_is_a_balanced_partition():
    for n in (0, 1, 7, 16, 31250):
        for world in (1, 2, 3, 8):
            parts = [sharding.shard(n, world, r) for r in range(world)]
            assert parts[0][0] == 0
            assert sum(c for _, c in parts) == n
            for (f0, c0), (f1, _) in zip(parts, parts[1:]):
                assert f0 + c0 == f1
            assert max(c for _, c in parts) - min(c for _, c in parts) <= 1
    with pytest.raises(ValueError):
        sharding.shard(10, 2, 2)


def _job():
    from difx_tests_b200 import synth
    return synth.make_job(nant=4, npol=2, nchan=128, numffts=96, bw=32e6, lo=1.4e9, rho=0.2, seed=3, nsubband=3)


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist

    from oracle import fxoracle as fo
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        job = _job()
        # time shards of subband 0
        f0, n = sharding.shard(job.numffts, world, rank)
        v, c = fo.correlate(job.data[0], job.delays, job.fileoffsets, job.bw, float(job.sb_lo[0]), job.nchan,
                            job.npol, fftindex=np.arange(f0, f0 + n), numffts=job.numffts,
                            maxoffset_ffts=job.numffts)
        vm, cm = sharding.merge_time_shards(v.astype(np.complex64), c)
        # subband shards
        s0, ns = sharding.shard(job.nsubband, world, rank)
        local = np.stack([fo.correlate(job.data[sb], job.delays, job.fileoffsets, job.bw, float(job.sb_lo[sb]),
                                       job.nchan, job.npol, numffts=job.numffts)[0].astype(np.complex64)
                          for sb in range(s0, s0 + ns)])
        allsb = sharding.gather_subbands(local, job.nsubband)
        tmax = sharding.max_over_ranks(1.5 + rank)
        q.put((rank, vm, cm, allsb, tmax))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_merge_time_and_subband_shards():
    from oracle import fxoracle as fo
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    job = _job()
    full, fc = fo.correlate(job.data[0], job.delays, job.fileoffsets, job.bw, float(job.sb_lo[0]), job.nchan,
                            job.npol, numffts=job.numffts)
    per_sb = np.stack([fo.correlate(job.data[sb], job.delays, job.fileoffsets, job.bw, float(job.sb_lo[sb]),
                                    job.nchan, job.npol, numffts=job.numffts)[0] for sb in range(job.nsubband)])
    for rank, vm, cm, allsb, tmax in results:
        np.testing.assert_array_equal(cm, fc)
        mx, _ = fo.vis_error(vm, full)
        assert mx.max() < 1e-6                     # two complex64 partial sums vs one
        assert allsb.shape == per_sb.shape
        assert fo.vis_error(allsb.reshape(-1, *per_sb.shape[2:]),
                            per_sb.reshape(-1, *per_sb.shape[2:]))[0].max() < 1e-6
        assert tmax == 2.5
