"""fxc_correlate_noalloc: the entry point for callers that cannot allocate
device memory when they correlate (a real-time path that must not touch the
allocator, or a host whose device memory another framework reserved up front).
It keeps every intermediate in the library's static scratch array, so the check
here is that two calls in a row -- the second reusing the scratch the first left
behind -- give the same visibilities and counts as the ordinary context path
(fxc_process_device + fxc_get_visibilities_device), and that a call leaves the
device's free memory unchanged.

Collected last on purpose: it must pass both alone in a fresh process and after
the other tests.  The test allocates its own output buffers (through torch);
only the entry point under test must not allocate."""
import ctypes as C

import numpy as np
import pytest

import difx_tests_b200 as fx
from difx_tests_b200 import synth
from oracle import fxoracle as fo

pytestmark = pytest.mark.gpu

VIS_TOL = 1e-5   # same bar as the plain-form parity tests


def _run_both(job, first_fft, nfft, check_free=False):
    import torch

    cfg = fx.make_config(job.nant, job.nchan, job.numffts, job.bw, job.lo, npol=job.npol, nsubband=job.nsubband)
    L = fx.lib()
    nvis = L.fxc_vis_count(C.byref(cfg))
    nout = job.nant * (job.nant - 1) // 2 + job.nant
    with fx.Correlator(cfg) as ctx:
        ctx.upload(job.data)
        dptr, pitch = ctx.device_input()
        # ordinary path
        ctx.process_device(dptr, pitch, job.delays, job.fileoffsets, first_fft, nfft)
        ref_vis, ref_counts = ctx.visibilities()
        # no-allocation path on the same device input, outputs owned by the caller
        d_vis = torch.zeros(2 * nvis, dtype=torch.float32, device="cuda")
        d_counts = torch.full((nout,), -1, dtype=torch.int32, device="cuda")
        stream = torch.cuda.current_stream()
        d = np.ascontiguousarray(job.delays, np.float64).reshape(-1)
        o = np.ascontiguousarray(job.fileoffsets, np.float64)
        def call():
            return L.fxc_correlate_noalloc(C.byref(cfg), C.c_void_p(dptr), pitch,
                                           d.ctypes.data_as(C.POINTER(C.c_double)),
                                           o.ctypes.data_as(C.POINTER(C.c_double)), first_fft, nfft,
                                           C.c_void_p(d_vis.data_ptr()), C.c_void_p(d_counts.data_ptr()), 0,
                                           C.c_void_p(stream.cuda_stream))
        st = call()
        assert st == fx.FXC_OK, L.fxc_strerror(st)
        torch.cuda.synchronize()
        if check_free:
            # after a first call (module loading, symbol lookup), a call allocates nothing:
            # the device's free memory (cudaMemGetInfo) is the same before and after it
            free0, _ = torch.cuda.mem_get_info()
            st = call()
            torch.cuda.synchronize()
            free1, _ = torch.cuda.mem_get_info()
            assert st == fx.FXC_OK, L.fxc_strerror(st)
            assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
        vis = d_vis.cpu().numpy().view(np.complex64).reshape(ref_vis.shape)
        counts = d_counts.cpu().numpy()
    return vis, counts, ref_vis, ref_counts


def test_noalloc_matches_context_path_twice_in_a_row():
    job_a = synth.make_job(nant=6, npol=2, nchan=256, numffts=96, bw=32e6, lo=1.4e9, rho=0.1, seed=501)
    job_b = synth.make_job(nant=9, npol=1, nchan=1024, numffts=80, bw=64e6, lo=1.65e9, rho=0.2, seed=502,
                           nsubband=2)
    for job, first, n, chk in ((job_a, 0, 96, False), (job_b, 7, 70, True)):
        vis, counts, ref_vis, ref_counts = _run_both(job, first, n, chk)
        np.testing.assert_array_equal(counts, ref_counts)
        mx, _ = fo.vis_error(vis, ref_vis)
        assert mx.max() < VIS_TOL, mx.max()
        assert np.abs(ref_vis).max() > 0


def test_noalloc_rejects_problems_beyond_its_scratch():
    # 64 antennas x 8 subbands x 1024 channels: accumulators alone exceed the scratch array
    cfg = fx.make_config(64, 1024, 64, 64e6, 1.4e9, npol=1, nsubband=8)
    d = np.zeros(3 * 64)
    o = np.zeros(64)
    L = fx.lib()
    st = L.fxc_correlate_noalloc(C.byref(cfg), C.c_void_p(256), 1 << 20, d.ctypes.data_as(C.POINTER(C.c_double)),
                                 o.ctypes.data_as(C.POINTER(C.c_double)), 0, 64, C.c_void_p(256), None, 0, None)
    assert st == fx.FXC_ERR_INVALID
