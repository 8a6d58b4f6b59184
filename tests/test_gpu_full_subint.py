"""Accumulation over a whole subintegration on the GPU against the FP64 oracle.

The reference sums every FFT of a subintegration into its FP32 visibilities (kernel.c:802,
829-854); the bench's geometry accumulates 31250 FFTs per subband.  Here one subband of
4 antennas x 1024 channels x 31250 FFTs (0.5 s at 128 MS/s) runs through each form, in the
library's own chunks, with the oracle accumulating in float64 over the same FFTs: the plain
FP32 form (on either FP32-grade F stage) stays within the plain bar of 1e-5 of max|V| per
spectrum, the FP16 tensor-core X form within its RMS bar.  A second case has the large-array
geometry (4096 channels, 2 polarisations, more than 128 signals: several 128 x 128 blocks of
the tensor-core Gram) over a few FFTs."""
import numpy as np
import pytest

import difx_tests_b200 as fx
from difx_tests_b200 import synth
from oracle import fxoracle as fo

pytestmark = pytest.mark.gpu

VIS_TOL = 1e-5
TC_RMS_TOL = 1e-3
TC_MAX_TOL = 1e-2


@pytest.fixture(scope="module")
def long_job():
    job = synth.make_long_job(nant=4, nchan=1024, numffts=31250, bw=64e6, lo=1.4e9, rho=0.1, seed=31)
    ref, rc = fo.correlate(job.data[0], job.delays, job.fileoffsets, job.bw, job.lo, job.nchan, 1,
                           numffts=job.numffts, maxoffset_ffts=job.numffts, chunk=1024)
    return job, ref, rc


def correlate(job, xmode, fstage):
    cfg = fx.make_config(job.nant, job.nchan, job.numffts, job.bw, job.lo, npol=1, xmode=xmode, fstage=fstage)
    with fx.Correlator(cfg) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        return c.visibilities()


@pytest.mark.parametrize("fstage", [fx.FXC_F_FFT32, fx.FXC_F_TC32])
def test_plain_form_over_a_full_subintegration(long_job, fstage):
    job, ref, rc = long_job
    vis, counts = correlate(job, fx.FXC_X_PLAIN_FP32, fstage)
    np.testing.assert_array_equal(counts, rc)
    assert rc.min() > 31000
    mx, rms = fo.vis_error(vis[0], ref)
    print(f"plain, fstage {fstage}: max {mx.max():.2e} rms {rms.max():.2e}")
    assert mx.max() < VIS_TOL, f"max {mx.max():.3e} rms {rms.max():.3e}"


@pytest.mark.parametrize("fstage", [fx.FXC_F_FFT32, fx.FXC_F_TC32, fx.FXC_F_TC16])
def test_tc_form_over_a_full_subintegration(long_job, fstage):
    job, ref, rc = long_job
    vis, counts = correlate(job, fx.FXC_X_TC_FP16, fstage)
    np.testing.assert_array_equal(counts, rc)
    mx, rms = fo.vis_error(vis[0], ref)
    print(f"tc, fstage {fstage}: max {mx.max():.2e} rms {rms.max():.2e}")
    assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL, f"max {mx.max():.3e} rms {rms.max():.3e}"


def test_large_array_geometry_several_gram_blocks():
    """72 antennas x 2 polarisations x 4096 channels, a few FFTs: 144 signals are 288 real rows of
    the Gram, three 128-row blocks (six block pairs per channel); FP16 tensor-core form vs FP64."""
    job = synth.make_job(nant=72, npol=2, nchan=4096, numffts=6, bw=64e6, lo=1.4e9, rho=0.02, seed=41)
    cfg = fx.make_config(job.nant, job.nchan, job.numffts, job.bw, job.lo, npol=2, xmode=fx.FXC_X_TC_FP16)
    with fx.Correlator(cfg) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    ref, rc = fo.correlate(job.data[0], job.delays, job.fileoffsets, job.bw, job.lo, job.nchan, 2,
                           numffts=job.numffts, maxoffset_ffts=job.numffts)
    np.testing.assert_array_equal(counts, rc)
    mx, rms = fo.vis_error(vis[0], ref)
    assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL, f"max {mx.max():.3e} rms {rms.max():.3e}"
