"""GPU parity of the FP16 tensor-core F stage (fxc_config.fstage = FXC_F_TC16; 2048-point
FFTs, one polarisation, F16 spectra): visibilities against the FP64 oracle at the tensor-core
bar, and against the FP32-FFT F stage (FXC_F_FFT32, the tensor-core forms' default).  Work
items are 16 FFTs of one (subband, antenna); the cases cover partial items (nfft not a multiple
of 16), several subbands, FFTs without data at the subintegration's edges and many items per
CTA."""
import numpy as np
import pytest

import difx_tests_b200 as fx
from difx_tests_b200 import synth
from oracle import fxoracle as fo

pytestmark = pytest.mark.gpu

TC_RMS_TOL = 1e-3    # RMS relative error per product spectrum vs FP64
TC_MAX_TOL = 1e-2    # max |d| / max |ref| per product spectrum


def corr_for(job, **kw):
    cfg = fx.make_config(job.nant, job.nchan, job.numffts, job.bw, job.lo, npol=job.npol, nsubband=job.nsubband,
                         sb_spacing=(job.sb_lo[1] - job.sb_lo[0]) if job.nsubband > 1 else job.bw, **kw)
    return fx.Correlator(cfg)


def run(job, monkeypatch, fstage=fx.FXC_F_TC16, **kw):
    with corr_for(job, fstage=fstage, **kw) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        return c.visibilities()


@pytest.mark.parametrize("nant,nsb,numffts,seed", [(8, 1, 64, 1), (16, 2, 200, 2), (40, 2, 517, 3)])
def test_tc_fstage_vs_fp64_oracle(nant, nsb, numffts, seed, monkeypatch):
    job = synth.make_job(nant=nant, npol=1, nchan=1024, numffts=numffts, bw=64e6, lo=1.4e9 + 0.25, rho=0.1,
                         seed=seed, nsubband=nsb)
    vis, counts = run(job, monkeypatch, xmode=fx.FXC_X_TC_FP16)
    worst = 0.0
    for sb in range(nsb):
        ref, rc = fo.correlate(job.data[sb], job.delays, job.fileoffsets, job.bw, float(job.sb_lo[sb]), job.nchan,
                               job.npol, numffts=job.numffts, maxoffset_ffts=job.numffts)
        np.testing.assert_array_equal(counts, rc)
        mx, rms = fo.vis_error(vis[sb], ref)
        worst = max(worst, rms.max())
        assert rms.max() < TC_RMS_TOL, f"sb {sb}: rms {rms.max():.3e}"
        assert mx.max() < TC_MAX_TOL, f"sb {sb}: max {mx.max():.3e}"
    print(f"tensor-core F stage: worst RMS {worst:.3e}")


def test_tc_fstage_matches_fft_fstage(monkeypatch):
    job = synth.make_job(nant=24, npol=1, nchan=1024, numffts=300, bw=64e6, lo=1.4e9, rho=0.1, seed=5)
    v_tc, c_tc = run(job, monkeypatch, xmode=fx.FXC_X_TC_FP16)
    v_fft, c_fft = run(job, monkeypatch, fstage=fx.FXC_F_FFT32, xmode=fx.FXC_X_TC_FP16)
    np.testing.assert_array_equal(c_tc, c_fft)
    mx, rms = fo.vis_error(v_tc[0], v_fft[0])
    assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL, f"rms {rms.max():.3e} max {mx.max():.3e}"


def test_tc_fstage_edge_ffts_without_data(monkeypatch):
    """Delays that push the first and last FFTs of some antennas outside the data: those
    FFTs contribute nothing, exactly as in the oracle (counts equal, visibilities close)."""
    job = synth.make_job(nant=6, npol=1, nchan=1024, numffts=48, bw=64e6, lo=1.4e9, rho=0.1, seed=9)
    job.fileoffsets[1] += 3.0 * 2048 / (2 * job.bw)     # antenna 1: data starts 3 FFTs late
    job.fileoffsets[4] -= 2.5 * 2048 / (2 * job.bw)     # antenna 4: runs off the end
    vis, counts = run(job, monkeypatch, xmode=fx.FXC_X_TC_FP16)
    ref, rc = fo.correlate(job.data[0], job.delays, job.fileoffsets, job.bw, job.lo, job.nchan, job.npol,
                           numffts=job.numffts, maxoffset_ffts=job.numffts)
    np.testing.assert_array_equal(counts, rc)
    assert rc.min() < job.numffts       # the case does have FFTs without data
    mx, rms = fo.vis_error(vis[0], ref)
    assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL, f"rms {rms.max():.3e} max {mx.max():.3e}"


def test_tc_fstage_fp8_form(monkeypatch):
    job = synth.make_job(nant=20, npol=1, nchan=1024, numffts=256, bw=64e6, lo=1.4e9, rho=0.1, seed=13)
    v8, c8 = run(job, monkeypatch, fstage=fx.FXC_F_TC16, xmode=fx.FXC_X_TC_FP8)
    v8f, c8f = run(job, monkeypatch, fstage=fx.FXC_F_FFT32, xmode=fx.FXC_X_TC_FP8)
    np.testing.assert_array_equal(c8, c8f)
    # the two F stages differ by FP16 rounding; the e4m3 quantisation of both dominates
    mx, rms = fo.vis_error(v8[0], v8f[0])
    assert rms.max() < 0.05, f"rms {rms.max():.3e}"


def test_tc_fstage_host_windows_equal_whole_device_input(monkeypatch):
    """Input streamed from the host through the three device windows gives exactly what the
    whole-subintegration device input gives (windows coincide with the spectra chunks)."""
    job = synth.make_job(nant=6, npol=1, nchan=1024, numffts=400, bw=64e6, lo=1.4e9, rho=0.1, seed=15, nsubband=2)
    with corr_for(job, fstage=fx.FXC_F_TC16, xmode=fx.FXC_X_TC_FP16, chunk_ffts=128) as c:
        c.upload(job.data)
        dptr, pitch = c.device_input()
        c.process_device(dptr, pitch, job.delays, job.fileoffsets)
        ref = c.visibilities()
        c.reset()
        c.process(job.data, job.delays, job.fileoffsets)
        got = c.visibilities()
    np.testing.assert_array_equal(got[1], ref[1])
    np.testing.assert_array_equal(got[0], ref[0])


def test_tc_fstage_window_only_context_vs_oracle(monkeypatch):
    job = synth.make_job(nant=5, npol=1, nchan=1024, numffts=300, bw=64e6, lo=1.4e9, rho=0.1, seed=17)
    job.fileoffsets[2] -= 20.3 * 2 * job.nchan / (2 * job.bw)   # its first FFTs have no data
    with corr_for(job, fstage=fx.FXC_F_TC16, xmode=fx.FXC_X_TC_FP16, chunk_ffts=128, window_ffts=70) as c:
        c.process_window(job.data, job.delays, job.fileoffsets, 11, 250)
        vis, counts = c.visibilities()
    ref, rc = fo.correlate(job.data[0], job.delays, job.fileoffsets, job.bw, job.lo, job.nchan, job.npol,
                           fftindex=np.arange(11, 261), numffts=job.numffts, maxoffset_ffts=job.numffts)
    np.testing.assert_array_equal(counts, rc)
    mx, rms = fo.vis_error(vis[0], ref)
    assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL, f"rms {rms.max():.3e} max {mx.max():.3e}"


def test_tc_fstage_subband_groups(monkeypatch):
    """A spectra budget too small for every subband: chunks over groups of subbands."""
    monkeypatch.setenv("FXC_SPECTRA_BUDGET_MB", "2")
    job = synth.make_job(nant=8, npol=1, nchan=1024, numffts=300, bw=64e6, lo=1.4e9, rho=0.1, seed=19, nsubband=3)
    vis, counts = run(job, monkeypatch, xmode=fx.FXC_X_TC_FP16)
    for sb in range(job.nsubband):
        ref, rc = fo.correlate(job.data[sb], job.delays, job.fileoffsets, job.bw, float(job.sb_lo[sb]), job.nchan,
                               job.npol, numffts=job.numffts, maxoffset_ffts=job.numffts)
        np.testing.assert_array_equal(counts, rc)
        mx, rms = fo.vis_error(vis[sb], ref)
        assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL, f"sb {sb}: rms {rms.max():.3e}"


def test_tensor_core_wait_expiry_is_reported_and_context_survives(monkeypatch):
    """The tensor-core kernels' bounded mbarrier wait, run out on a barrier that nothing
    completes, comes back as FXC_ERR_TIMEOUT with code 7; the next tensor-core correlation on
    the same context is correct."""
    import ctypes as C
    job = synth.make_job(nant=6, npol=1, nchan=1024, numffts=64, bw=64e6, lo=1.4e9, rho=0.1, seed=23)
    with corr_for(job, fstage=fx.FXC_F_TC16, xmode=fx.FXC_X_TC_FP16) as c:
        assert fx.lib().fxc_debug_expire_wait_tc(C.c_void_p(c.handle.value)) == fx.FXC_OK
        with pytest.raises(fx.FxcError) as e:
            c.synchronize()
        assert e.value.status == fx.FXC_ERR_TIMEOUT
        assert fx.lib().fxc_last_device_error() == 7
        c.reset()
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    ref, rc = fo.correlate(job.data[0], job.delays, job.fileoffsets, job.bw, job.lo, job.nchan, job.npol,
                           numffts=job.numffts, maxoffset_ffts=job.numffts)
    np.testing.assert_array_equal(counts, rc)
    mx, rms = fo.vis_error(vis[0], ref)
    assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL
