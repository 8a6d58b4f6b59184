"""GPU parity of the FP32-grade tensor-core F stage (fxc_config.fstage = FXC_F_TC32; 2048-point
FFTs, one polarisation): the 32 x 64 DFT as two tcgen05 GEMMs whose FP16 operands are
error-compensated pairs (three products per GEMM, FP32 accumulation).

It is held to the FP32 F stage's bars, not the FP16 ones: spectra within 2e-5 of max|X| per
spectrum of the FP64 oracle (the FP32 FFT's bar), and with the plain FP32 X stage visibilities
within 1e-5 of max|V| per spectrum of the FP64 oracle (the plain form's bar).  With the FP16
tensor-core X stage the visibilities meet the tensor-core bar and agree with the FP32-FFT F
stage's to within the X stage's own FP16 rounding.  Work items are 8 FFTs of one (subband,
antenna); the cases cover partial items, several subbands, FFTs without data at the
subintegration's edges, windows and many items per CTA."""
import numpy as np
import pytest

import difx_tests_b200 as fx
from difx_tests_b200 import synth
from oracle import fxoracle as fo

pytestmark = pytest.mark.gpu

SPEC_TOL = 2e-5      # FP32 F stage vs FP64 oracle, relative to max|X| per spectrum
VIS_TOL = 1e-5       # plain FP32 form vs FP64 oracle, relative to max|V| per spectrum
TC_RMS_TOL = 1e-3    # FP16 tensor-core X form: RMS relative error per product spectrum vs FP64
TC_MAX_TOL = 1e-2


def corr_for(job, **kw):
    cfg = fx.make_config(job.nant, job.nchan, job.numffts, job.bw, job.lo, npol=job.npol, nsubband=job.nsubband,
                         sb_spacing=(job.sb_lo[1] - job.sb_lo[0]) if job.nsubband > 1 else job.bw,
                         fstage=kw.pop("fstage", fx.FXC_F_TC32), **kw)
    return fx.Correlator(cfg)


def run(job, **kw):
    with corr_for(job, **kw) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        return c.visibilities()


def oracle_vis(job, sb=0, fftindex=None):
    return fo.correlate(job.data[sb], job.delays, job.fileoffsets, job.bw, float(job.sb_lo[sb]), job.nchan,
                        job.npol, fftindex=fftindex, numffts=job.numffts, maxoffset_ffts=job.numffts)


@pytest.mark.parametrize("nf,seed", [(24, 1), (61, 2)])
def test_tc32_spectra_meet_the_fp32_bar(nf, seed):
    job = synth.random_job(nant=3, npol=1, nchan=1024, numffts=nf, bw=64e6, lo=1.4e9 + 0.3, seed=seed)
    with corr_for(job) as c:
        got = c.spectra(job.data, job.delays, job.fileoffsets, 0, nf)[0]          # [sig][t][C]
    spec, tab = fo.channelise(job.data[0], job.delays, job.fileoffsets, job.bw, job.lo, 1024, 1, np.arange(nf), nf)
    ref = spec.reshape(job.nant, nf, 1024)
    err = np.abs(got - ref).max(axis=-1) / np.maximum(np.abs(ref).max(axis=-1), 1e-30)
    valid = tab["valid"]
    print(f"tc32 spectra: worst {err[valid].max():.2e}")
    assert err[valid].max() < SPEC_TOL, err[valid].max()
    assert np.all(got[~valid] == 0)


@pytest.mark.parametrize("nant,nsb,numffts,seed", [(4, 1, 40, 3), (12, 2, 203, 4)])
def test_tc32_with_plain_x_meets_the_plain_bar(nant, nsb, numffts, seed):
    job = synth.make_job(nant=nant, npol=1, nchan=1024, numffts=numffts, bw=64e6, lo=1.4e9 + 0.25, rho=0.1,
                         seed=seed, nsubband=nsb)
    vis, counts = run(job, xmode=fx.FXC_X_PLAIN_FP32)
    for sb in range(nsb):
        ref, rc = oracle_vis(job, sb)
        np.testing.assert_array_equal(counts, rc)
        mx, rms = fo.vis_error(vis[sb], ref)
        assert mx.max() < VIS_TOL, f"sb {sb}: max {mx.max():.3e} rms {rms.max():.3e}"


@pytest.mark.parametrize("nant,nsb,numffts,seed", [(8, 1, 64, 5), (40, 2, 517, 6)])
def test_tc32_with_tc_x_vs_fp64_oracle(nant, nsb, numffts, seed):
    job = synth.make_job(nant=nant, npol=1, nchan=1024, numffts=numffts, bw=64e6, lo=1.4e9 + 0.25, rho=0.1,
                         seed=seed, nsubband=nsb)
    vis, counts = run(job, xmode=fx.FXC_X_TC_FP16)
    for sb in range(nsb):
        ref, rc = oracle_vis(job, sb)
        np.testing.assert_array_equal(counts, rc)
        mx, rms = fo.vis_error(vis[sb], ref)
        assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL, f"sb {sb}: rms {rms.max():.3e} max {mx.max():.3e}"


def test_tc32_matches_the_fft_fstage_through_the_tc_x_stage():
    """Both F stages are FP32-grade, so behind the same FP16 X stage the two correlations differ
    only where an FP16 cast of a spectrum value rounds differently."""
    job = synth.make_job(nant=24, npol=1, nchan=1024, numffts=300, bw=64e6, lo=1.4e9, rho=0.1, seed=7)
    v32, c32 = run(job, xmode=fx.FXC_X_TC_FP16)
    vff, cff = run(job, xmode=fx.FXC_X_TC_FP16, fstage=fx.FXC_F_FFT32)
    np.testing.assert_array_equal(c32, cff)
    mx, rms = fo.vis_error(v32[0], vff[0])
    assert rms.max() < 1e-4, f"rms {rms.max():.3e} max {mx.max():.3e}"


def test_tc32_edge_ffts_without_data():
    job = synth.make_job(nant=6, npol=1, nchan=1024, numffts=45, bw=64e6, lo=1.4e9, rho=0.1, seed=9)
    job.fileoffsets[1] += 3.0 * 2048 / (2 * job.bw)     # antenna 1: data starts 3 FFTs late
    job.fileoffsets[4] -= 2.5 * 2048 / (2 * job.bw)     # antenna 4: runs off the end
    vis, counts = run(job, xmode=fx.FXC_X_PLAIN_FP32)
    ref, rc = oracle_vis(job)
    np.testing.assert_array_equal(counts, rc)
    assert rc.min() < job.numffts
    mx, rms = fo.vis_error(vis[0], ref)
    assert mx.max() < VIS_TOL, f"max {mx.max():.3e}"


def test_tc32_window_only_context_vs_oracle():
    job = synth.make_job(nant=5, npol=1, nchan=1024, numffts=300, bw=64e6, lo=1.4e9, rho=0.1, seed=17)
    job.fileoffsets[2] -= 20.3 * 2 * job.nchan / (2 * job.bw)   # its first FFTs have no data
    with corr_for(job, xmode=fx.FXC_X_TC_FP16, chunk_ffts=128, window_ffts=70) as c:
        c.process_window(job.data, job.delays, job.fileoffsets, 11, 250)
        vis, counts = c.visibilities()
    ref, rc = oracle_vis(job, fftindex=np.arange(11, 261))
    np.testing.assert_array_equal(counts, rc)
    mx, rms = fo.vis_error(vis[0], ref)
    assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL, f"rms {rms.max():.3e} max {mx.max():.3e}"


def test_tc32_fp8_form_matches_the_fft_fstage():
    """The FP8 form's per-(channel, signal) absmax comes from the output warps of the tensor-core F
    stage: the e4m3 correlation equals the one on the FP32 FFT F stage up to the quantisation."""
    job = synth.make_job(nant=20, npol=1, nchan=1024, numffts=256, bw=64e6, lo=1.4e9, rho=0.1, seed=13)
    v32, c32 = run(job, xmode=fx.FXC_X_TC_FP8)
    vff, cff = run(job, xmode=fx.FXC_X_TC_FP8, fstage=fx.FXC_F_FFT32)
    np.testing.assert_array_equal(c32, cff)
    mx, rms = fo.vis_error(v32[0], vff[0])
    assert rms.max() < 0.05, f"rms {rms.max():.3e}"
    ref, rc = oracle_vis(job)
    mx, rms = fo.vis_error(v32[0], ref)
    assert rms.max() < 0.1, f"vs FP64: rms {rms.max():.3e}"


def test_tc32_rejected_where_it_does_not_apply():
    for kw in (dict(nchan=512, npol=1, xmode=fx.FXC_X_TC_FP16), dict(nchan=1024, npol=2, xmode=fx.FXC_X_TC_FP16),
               dict(nchan=2048, npol=1, xmode=fx.FXC_X_PLAIN_FP32)):
        cfg = fx.make_config(4, kw["nchan"], 64, 64e6, 1.4e9, npol=kw["npol"], xmode=kw["xmode"],
                             fstage=fx.FXC_F_TC32)
        with pytest.raises(fx.FxcError) as e:
            fx.Correlator(cfg)
        assert e.value.status == fx.FXC_ERR_UNSUPPORTED
