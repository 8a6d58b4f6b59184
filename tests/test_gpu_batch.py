"""Multi-job batch (fxc_batch_*): many uneven jobs in grouped persistent launches.

Every job of a batch must give exactly what the single-job plain path gives for
the same inputs (the same kernels run per FFT and per channel, in the same
accumulation order), whatever FFT block size or X tile variant the autotuner
picks, eagerly or replayed from the CUDA graph; and within 1e-5 of the FP64
oracle.
"""
import numpy as np
import pytest

import difx_tests_b200 as fx
from difx_tests_b200 import synth
from oracle import fxoracle as fo

pytestmark = pytest.mark.gpu

VIS_TOL = 1e-5

# uneven jobs: antennas 4..56, FFT lengths 256..8192, 1..8 subbands, 1 or 2 polarisations,
# several spectra chunks for some (chunk_ffts) so rounds differ between jobs
JOBS = [
    dict(nant=4, npol=2, nchan=128, nsubband=3, numffts=300, chunk_ffts=64),
    dict(nant=13, npol=1, nchan=1024, nsubband=1, numffts=150),
    dict(nant=7, npol=2, nchan=4096, nsubband=2, numffts=40),
    dict(nant=30, npol=1, nchan=256, nsubband=2, numffts=200, chunk_ffts=128),
    dict(nant=4, npol=2, nchan=128, nsubband=1, numffts=90),
    dict(nant=56, npol=1, nchan=512, nsubband=1, numffts=64),
    dict(nant=5, npol=1, nchan=2048, nsubband=8, numffts=33),
]


def make_jobs():
    jobs, cfgs = [], []
    for i, p in enumerate(JOBS):
        j = synth.random_job(nant=p["nant"], npol=p["npol"], nchan=p["nchan"], numffts=p["numffts"], bw=32e6,
                             seed=100 + i, nsubband=p["nsubband"])
        jobs.append(j)
        cfgs.append(fx.make_config(j.nant, j.nchan, j.numffts, j.bw, j.lo, npol=j.npol, nsubband=j.nsubband,
                                   sb_spacing=j.bw, chunk_ffts=p.get("chunk_ffts", 0)))
    return jobs, cfgs


def single(job, cfg):
    with fx.Correlator(cfg) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        return c.visibilities()


@pytest.fixture(scope="module")
def jobs_and_refs():
    jobs, cfgs = make_jobs()
    refs = [single(j, c) for j, c in zip(jobs, cfgs)]
    return jobs, cfgs, refs


def load(b, jobs):
    for i, j in enumerate(jobs):
        b.upload(i, j.data)
        b.set_model(i, j.delays, j.fileoffsets)


def test_batch_equals_single_job_path(jobs_and_refs):
    jobs, cfgs, refs = jobs_and_refs
    with fx.Batch(cfgs) as b:
        load(b, jobs)
        b.process()                      # eager
        for i in range(len(jobs)):
            vis, counts = b.visibilities(i)
            np.testing.assert_array_equal(counts, refs[i][1])
            np.testing.assert_array_equal(vis, refs[i][0])
        b.reset()
        b.process()                      # captured
        b.reset()
        b.process()                      # replayed
        for i in range(len(jobs)):
            vis, counts = b.visibilities(i)
            np.testing.assert_array_equal(counts, refs[i][1])
            np.testing.assert_array_equal(vis, refs[i][0])


@pytest.mark.parametrize("i", [0, 2, 6])
def test_batch_vs_oracle(jobs_and_refs, i):
    jobs, cfgs, refs = jobs_and_refs
    j = jobs[i]
    for sb in range(j.nsubband):
        ref = fo.correlate(j.data[sb], j.delays, j.fileoffsets, j.bw, float(j.sb_lo[sb]), j.nchan, j.npol,
                           numffts=j.numffts, maxoffset_ffts=j.numffts)[0]
        mx, rms = fo.vis_error(refs[i][0][sb], ref)
        assert mx.max() < VIS_TOL, f"job {i} sb {sb}: {mx.max():.3e}"


def test_autotune_keeps_results_and_writes_plan_cache(jobs_and_refs, tmp_path, monkeypatch):
    jobs, cfgs, refs = jobs_and_refs
    cache = tmp_path / "plans.txt"
    monkeypatch.setenv("FXC_PLAN_CACHE", str(cache))
    with fx.Batch(cfgs) as b:
        load(b, jobs)
        b.autotune(reps=2)
        plans = [b.plan(i) for i in range(len(jobs))]
        assert all(tb in (8, 16, 32) and alt in (0, 1) for tb, alt in plans)
        for _ in range(2):               # eager, then captured with the tuned plans
            b.reset()
            b.process()
        for i in range(len(jobs)):
            vis, counts = b.visibilities(i)
            np.testing.assert_array_equal(vis, refs[i][0])
    text = cache.read_text().split("\n")
    assert any(line.startswith("F 256 2 ") for line in text)
    # a new batch picks the cached plans up
    with fx.Batch(cfgs) as b2:
        assert [b2.plan(i) for i in range(len(jobs))] == plans


def test_model_change_between_replays(jobs_and_refs):
    jobs, cfgs, refs = jobs_and_refs
    with fx.Batch(cfgs[:3]) as b:
        load(b, jobs[:3])
        b.process()
        b.reset()
        b.process()                      # graph recorded
        j = jobs[1]
        d = j.delays.copy()
        d[:, 0] += 3.7e-7
        b.set_model(1, d, j.fileoffsets)
        b.reset()
        b.process()                      # replay sees the new model
        vis, _ = b.visibilities(1)
        with fx.Correlator(cfgs[1]) as c:
            c.process(j.data, d, j.fileoffsets)
            np.testing.assert_array_equal(vis, c.visibilities()[0])
        np.testing.assert_array_equal(b.visibilities(0)[0], refs[0][0])


def test_graph_off_matches(jobs_and_refs):
    jobs, cfgs, refs = jobs_and_refs
    with fx.Batch(cfgs[3:]) as b:
        b.use_graph(False)
        load(b, jobs[3:])
        b.process()
        b.reset()
        b.process()
        for k in range(len(jobs) - 3):
            np.testing.assert_array_equal(b.visibilities(k)[0], refs[3 + k][0])


# mixed batch: FP16 tensor-core jobs (their spectra from a grouped F16 F-stage launch, their X
# stage its own launch inside the graph) and a plain job of more than 64 signals beside plain
# grouped jobs
MIXED = [
    dict(nant=6, npol=1, nchan=1024, nsubband=2, numffts=150, xmode=fx.FXC_X_TC_FP16),
    dict(nant=40, npol=2, nchan=256, nsubband=1, numffts=96, xmode=fx.FXC_X_PLAIN_FP32),   # 80 signals
    dict(nant=9, npol=1, nchan=1024, nsubband=1, numffts=200, xmode=fx.FXC_X_PLAIN_FP32),
    dict(nant=20, npol=2, nchan=512, nsubband=1, numffts=64, xmode=fx.FXC_X_TC_FP16),
]
TC_RMS_TOL = 1e-3


def test_mixed_batch_tc_and_large_jobs_vs_oracle():
    jobs, cfgs = [], []
    for i, p in enumerate(MIXED):
        j = synth.make_job(nant=p["nant"], npol=p["npol"], nchan=p["nchan"], numffts=p["numffts"], bw=32e6,
                           lo=1.4e9, rho=0.1, seed=300 + i, nsubband=p["nsubband"])
        jobs.append(j)
        cfgs.append(fx.make_config(j.nant, j.nchan, j.numffts, j.bw, j.lo, npol=j.npol, nsubband=j.nsubband,
                                   sb_spacing=j.bw, xmode=p["xmode"]))
    with fx.Batch(cfgs) as b:
        load(b, jobs)
        for _ in range(3):               # eager, captured, replayed
            b.reset()
            b.process()
        for i, (j, p) in enumerate(zip(jobs, MIXED)):
            vis, counts = b.visibilities(i)
            for sb in range(j.nsubband):
                ref, rc = fo.correlate(j.data[sb], j.delays, j.fileoffsets, j.bw, float(j.sb_lo[sb]), j.nchan,
                                       j.npol, numffts=j.numffts, maxoffset_ffts=j.numffts)
                np.testing.assert_array_equal(counts, rc)
                mx, rms = fo.vis_error(vis[sb], ref)
                if p["xmode"] == fx.FXC_X_TC_FP16:
                    assert rms.max() < TC_RMS_TOL, f"job {i} sb {sb}: rms {rms.max():.3e}"
                else:
                    assert mx.max() < VIS_TOL, f"job {i} sb {sb}: max {mx.max():.3e}"
        b.autotune(reps=1)               # F16 groups only try blocks whose staging fits
        b.reset()
        b.process()
        vis, _ = b.visibilities(0)
        with fx.Correlator(cfgs[0]) as c:
            c.process(jobs[0].data, jobs[0].delays, jobs[0].fileoffsets)
            mx, rms = fo.vis_error(vis[0], c.visibilities()[0][0])
        assert rms.max() < 1e-5          # same F16 spectra, chunked differently: accumulation order only
