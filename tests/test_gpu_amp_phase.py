"""Amplitude and phase of the visibilities computed on the device (fxc_get_amp_phase), the two
columns the reference's saveVisibilities prints beside re and im (kernel.c:594-596,
vectorMagnitude / vectorPhase), against the same quantities computed in FP64 from the
visibilities the library returns."""
import numpy as np
import pytest

import difx_tests_b200 as fx
from difx_tests_b200 import synth


@pytest.mark.gpu
@pytest.mark.parametrize("npol,nsb,normalize", [(1, 1, True), (2, 2, False)])
def test_amp_phase_match_the_visibilities(npol, nsb, normalize):
    job = synth.make_job(nant=5, npol=npol, nchan=256, numffts=96, bw=32e6, lo=1.4e9, rho=0.1, seed=21, nsubband=nsb)
    cfg = fx.make_config(job.nant, job.nchan, job.numffts, job.bw, job.lo, npol=npol, nsubband=nsb)
    with fx.Correlator(cfg) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, _ = c.visibilities(normalize=normalize)
        amp, ph = c.amp_phase(normalize=normalize)
    v = vis.astype(np.complex128)
    ref_amp = np.abs(v)
    scale = ref_amp.max()
    # |v|: the sum of squares rounded once more than FP64, relative to the spectrum scale
    assert np.abs(amp - ref_amp).max() <= 2e-7 * scale
    # phase: FP32 atan2 of the same FP32 pair (a few ulp of pi); near-zero values excepted
    big = ref_amp > 1e-4 * scale
    d = np.angle(np.exp(1j * (ph.astype(np.float64) - np.angle(v))))
    assert np.abs(d[big]).max() <= 2e-6
    assert np.all(np.abs(ph) <= np.float32(np.pi))
