"""Time and subband shards of one subintegration correlated through the library by two
processes, merged over torch.distributed, against one process correlating it whole.

The reference splits a subintegration's FFTs into `split` partial accumulations and sums them
(main.c:398-433, kernel.c:856-878); sharding.correlate_shard does that across ranks (time
shards: one all-reduce of visibilities and counts) or hands each rank whole subbands (one
all-gather).  The test runs on one GPU, so both ranks share it: their kernels are
independent (nothing on the device waits on the other rank) and the collectives run on the
host through gloo; under NCCL the same code keeps the buffers on the device."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NSB, NANT, NCHAN, NFFT = 3, 5, 256, 200


def _job():
    from difx_tests_b200 import synth
    return synth.make_job(nant=NANT, npol=1, nchan=NCHAN, numffts=NFFT, bw=32e6, lo=1.4e9, rho=0.2, seed=71,
                          nsubband=NSB)


def _device_rows(torch, job, fx, cfg):
    subint = fx.lib().fxc_subint_bytes(cfg)
    pitch = (subint + 16 + 255) // 256 * 256
    rows = np.zeros((NSB * NANT, pitch), np.uint8)
    rows[:, :subint] = job.data.reshape(NSB * NANT, -1)[:, :subint]
    return torch.from_numpy(rows).cuda(), pitch


def _rank_main(rank, world, port, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch
    import torch.distributed as dist

    import difx_tests_b200 as fx
    from difx_tests_b200 import sharding
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        torch.cuda.set_device(0)
        job = _job()
        cfg = fx.make_config(NANT, NCHAN, NFFT, job.bw, job.lo, npol=1, nsubband=NSB, sb_spacing=job.bw)
        d, pitch = _device_rows(torch, job, fx, cfg)
        rcfg, f0, n, s0 = sharding.shard_config(fx, cfg, mode, world, rank)
        with fx.Correlator(rcfg) as corr:
            vis, counts = sharding.correlate_shard(fx, corr, mode, d.data_ptr(), pitch, job.delays, job.fileoffsets,
                                                   f0, n, s0, NSB, torch.device("cuda", 0))
        q.put((rank, vis.cpu().numpy(), counts.numpy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("mode", ["time", "subband"])
def test_two_ranks_merge_to_the_whole_correlation(mode):
    import difx_tests_b200 as fx
    from oracle import fxoracle as fo
    job = _job()
    cfg = fx.make_config(NANT, NCHAN, NFFT, job.bw, job.lo, npol=1, nsubband=NSB, sb_spacing=job.bw)
    with fx.Correlator(cfg) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        whole, wc = c.visibilities()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, vis, counts in results:
        got = vis.view(np.complex64).reshape(whole.shape)
        np.testing.assert_array_equal(counts, wc)
        for sb in range(NSB):
            mx, _ = fo.vis_error(got[sb], whole[sb])
            # time shards add two FP32 partial sums instead of accumulating one: rounding only
            assert mx.max() < 1e-6, (rank, sb, mx.max())
