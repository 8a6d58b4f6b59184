"""8-bit complex input (the reference's GPU-path sample format): int8 (re, im) per
sample and polarisation, FFT length nchan, every bin a channel.  The CUDA path
against the FP64 oracle's restatement of that format: spectra within 2e-5,
plain visibilities within 1e-5, tensor-core forms within their bars."""
import numpy as np
import pytest

import difx_tests_b200 as fx
from difx_tests_b200 import synth
from oracle import fxoracle as fo

pytestmark = pytest.mark.gpu

SPEC_TOL = 2e-5
VIS_TOL = 1e-5


def cfg_for(job, **kw):
    return fx.make_config(job.nant, job.nchan, job.numffts, job.bw, job.lo, npol=job.npol, nsubband=job.nsubband,
                          sb_spacing=job.bw, cpx=True, **kw)


def oracle(job, sb=0, **kw):
    return fo.correlate(job.data[sb], job.delays, job.fileoffsets, job.bw, float(job.sb_lo[sb]), job.nchan,
                        job.npol, numffts=job.numffts, maxoffset_ffts=job.numffts, cpx=True, **kw)


@pytest.mark.parametrize("npol,nchan", [(1, 256), (2, 512), (1, 1024), (2, 2048), (2, 4096)])
def test_complex_spectra_vs_oracle(npol, nchan):
    job = synth.random_job(nant=3, npol=npol, nchan=nchan, numffts=24, bw=32e6, seed=nchan + npol, cpx=True)
    job.fileoffsets[1] += 1.0 / job.bw          # whole-sample shifts of the window
    job.fileoffsets[2] += 7.3 / job.bw
    with fx.Correlator(cfg_for(job)) as c:
        got = c.spectra(job.data, job.delays, job.fileoffsets, 0, job.numffts)[0]   # [sig][t][chan]
    ref, tab = fo.channelise(job.data[0], job.delays, job.fileoffsets, job.bw, job.lo, job.nchan, job.npol,
                             np.arange(job.numffts), job.numffts, cpx=True)
    ref = ref.reshape(job.nant * job.npol, job.numffts, job.nchan)
    scale = np.abs(ref).max(axis=-1, keepdims=True)
    scale[scale == 0] = 1
    assert (np.abs(got - ref) / scale).max() < SPEC_TOL


@pytest.mark.parametrize("nant,npol,nchan,nsb", [(4, 2, 256, 1), (6, 1, 1024, 2), (3, 2, 4096, 1)])
def test_complex_vis_plain_vs_oracle(nant, npol, nchan, nsb):
    job = synth.random_job(nant=nant, npol=npol, nchan=nchan, numffts=100, bw=64e6, seed=nant * nchan,
                           nsubband=nsb, cpx=True)
    with fx.Correlator(cfg_for(job, chunk_ffts=64)) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    for sb in range(nsb):
        ref, rc = oracle(job, sb)
        np.testing.assert_array_equal(counts, rc)
        mx, rms = fo.vis_error(vis[sb], ref)
        assert mx.max() < VIS_TOL, f"sb {sb}: {mx.max():.3e}"


@pytest.mark.parametrize("xmode", [fx.FXC_X_TC_FP16, fx.FXC_X_TC_FP8])
def test_complex_tensor_core_forms(xmode):
    job = synth.random_job(nant=20, npol=2, nchan=1024, numffts=128, bw=64e6, seed=77, cpx=True)
    with fx.Correlator(cfg_for(job, xmode=xmode)) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    ref, rc = oracle(job)
    np.testing.assert_array_equal(counts, rc)
    mx, rms = fo.vis_error(vis[0], ref)
    if xmode == fx.FXC_X_TC_FP16:
        # uncorrelated random samples: |V| of a cross spectrum is only ~sqrt(N) sigma^2, so the
        # F16 rounding (2^-11 per value, both factors) reaches ~7e-4 of it; bar 2e-3
        assert rms.max() < 2e-3 and mx.max() < 1e-2
    else:
        assert rms.max() < 0.05


def test_complex_windows_and_time_shards():
    job = synth.random_job(nant=5, npol=1, nchan=512, numffts=300, bw=64e6, seed=8, cpx=True)
    with fx.Correlator(cfg_for(job, window_ffts=70)) as c:
        c.process_window(job.data, job.delays, job.fileoffsets, 0, 150)
        c.process_window(job.data, job.delays, job.fileoffsets, 150, 150)
        vis, counts = c.visibilities()
    ref, rc = oracle(job)
    np.testing.assert_array_equal(counts, rc)
    assert fo.vis_error(vis[0], ref)[0].max() < VIS_TOL
