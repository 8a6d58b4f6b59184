"""Streamed input: host subintegrations copied window by window (three device
windows, copies on their own stream), explicit device windows, and the
coverage check that keeps an FFT from reading outside its window.

The windowed host path must give exactly what the whole-subintegration device
path gives when its windows coincide with the spectra chunks, and match the
FP64 oracle within the plain-form bar otherwise.
"""
import numpy as np
import pytest

import difx_tests_b200 as fx
from difx_tests_b200 import synth
from oracle import fxoracle as fo

pytestmark = pytest.mark.gpu

VIS_TOL = 1e-5


def cfg_for(job, **kw):
    return fx.make_config(job.nant, job.nchan, job.numffts, job.bw, job.lo, npol=job.npol, nsubband=job.nsubband,
                          sb_spacing=job.bw, **kw)


def oracle(job, sb=0):
    return fo.correlate(job.data[sb], job.delays, job.fileoffsets, job.bw, float(job.sb_lo[sb]), job.nchan,
                        job.npol, numffts=job.numffts, maxoffset_ffts=job.numffts)


@pytest.mark.parametrize("xmode", [fx.FXC_X_PLAIN_FP32, fx.FXC_X_TC_FP16])
def test_host_windows_equal_whole_device_input(xmode):
    job = synth.make_job(nant=6, npol=2, nchan=256, numffts=700, bw=64e6, lo=1.4e9, rho=0.1, seed=5, nsubband=2)
    with fx.Correlator(cfg_for(job, xmode=xmode, chunk_ffts=128)) as c:
        c.upload(job.data)
        dptr, pitch = c.device_input()
        c.process_device(dptr, pitch, job.delays, job.fileoffsets)
        ref = c.visibilities()
        c.reset()
        c.process(job.data, job.delays, job.fileoffsets)       # windows of one chunk each
        got = c.visibilities()
    np.testing.assert_array_equal(got[1], ref[1])
    np.testing.assert_array_equal(got[0], ref[0])


@pytest.mark.parametrize("window_ffts,first,nfft", [(100, 0, 500), (37, 13, 300), (500, 0, 500)])
def test_window_only_context_vs_oracle(window_ffts, first, nfft):
    job = synth.make_job(nant=5, npol=1, nchan=512, numffts=500, bw=64e6, lo=1.4e9, rho=0.1, seed=9)
    # one antenna far from its file offset: 40.3 FFTs of net delay, so its first FFTs are invalid
    job.fileoffsets[2] -= 40.3 * 2 * job.nchan / (2 * job.bw)
    with fx.Correlator(cfg_for(job, chunk_ffts=128, window_ffts=window_ffts)) as c:
        with pytest.raises(fx.FxcError):
            c.upload(job.data)                                  # no whole-subintegration buffer
        c.process_window(job.data, job.delays, job.fileoffsets, first, nfft)
        vis, counts = c.visibilities()
    ref, rc = fo.correlate(job.data[0], job.delays, job.fileoffsets, job.bw, job.lo, job.nchan, job.npol,
                           fftindex=np.arange(first, first + nfft), numffts=job.numffts,
                           maxoffset_ffts=job.numffts)
    np.testing.assert_array_equal(counts, rc)
    mx, rms = fo.vis_error(vis[0], ref)
    assert mx.max() < VIS_TOL


def test_device_windows_and_miss_detection():
    import torch

    job = synth.make_job(nant=4, npol=2, nchan=256, numffts=400, bw=64e6, lo=1.4e9, rho=0.1, seed=13)
    F = 2 * job.nchan
    spb = 4 // job.npol
    cfg = cfg_for(job, chunk_ffts=64, window_ffts=64)
    ref, rc = oracle(job)
    with fx.Correlator(cfg) as c:
        # two device windows of 200 FFTs each, every antenna's window starting 3 FFTs early
        for w0 in (0, 200):
            base = np.full(job.nant, max(0, (w0 - 3) * F), np.int64)
            base -= base % spb
            nbytes = (206 * F) // spb
            rows = np.zeros((job.nant, nbytes + 64), np.uint8)
            for a in range(job.nant):
                src = job.data[0, a, base[a] // spb: base[a] // spb + nbytes]
                rows[a, :src.size] = src
            d = torch.from_numpy(rows).cuda()
            torch.cuda.synchronize()
            c.process_device_window(d.data_ptr(), rows.shape[1], base, nbytes, job.delays, job.fileoffsets, w0, 200)
            c.synchronize()
            del d
        vis, counts = c.visibilities()
        np.testing.assert_array_equal(counts, rc)
        assert fo.vis_error(vis[0], ref)[0].max() < VIS_TOL
        # a window that misses the FFTs' samples: reported, nothing read outside the rows
        c.reset()
        rows = np.zeros((job.nant, 10 * F // spb + 64), np.uint8)
        d = torch.from_numpy(rows).cuda()
        torch.cuda.synchronize()
        c.process_device_window(d.data_ptr(), rows.shape[1], np.zeros(job.nant, np.int64), 10 * F // spb,
                                job.delays, job.fileoffsets, 100, 50)
        with pytest.raises(fx.FxcError) as e:
            c.synchronize()
        assert e.value.status == fx.FXC_ERR_INVALID
        c.synchronize()      # the error is reported once; the context stays usable


@pytest.mark.parametrize("xmode", [fx.FXC_X_PLAIN_FP32, fx.FXC_X_TC_FP16, fx.FXC_X_TC_FP8])
def test_subband_groups(xmode, monkeypatch):
    """A spectra budget too small for every subband: chunks over groups of subbands."""
    monkeypatch.setenv("FXC_SPECTRA_BUDGET_MB", "1")
    job = synth.make_job(nant=8, npol=1, nchan=512, numffts=600, bw=64e6, lo=1.4e9, rho=0.1, seed=21, nsubband=3)
    with fx.Correlator(cfg_for(job, xmode=xmode)) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    for sb in range(job.nsubband):
        ref, rc = oracle(job, sb)
        np.testing.assert_array_equal(counts, rc)
        mx, rms = fo.vis_error(vis[sb], ref)
        if xmode == fx.FXC_X_PLAIN_FP32:
            assert mx.max() < VIS_TOL
        elif xmode == fx.FXC_X_TC_FP16:
            assert rms.max() < 1e-3 and mx.max() < 1e-2
        else:
            assert rms.max() < 0.05
