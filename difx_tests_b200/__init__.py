"""B200 (sm_100a) FX correlator hot path behind a C ABI.

``libfxcorr.so`` (built from ``difx_tests_b200/csrc`` into
``difx_tests_b200/lib``) implements the reference's per-subintegration
processing (twiG56/difx_tests kernel.c: unpack, integer/fractional delay,
fringe rotation, FFT, fractional-sample correction, cross-multiply-accumulate)
on one GPU.  This module is a thin ctypes binding of ``include/fxcorr.h``; it
never computes anything on the CPU and raises if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libfxcorr.so")
REPO = os.path.dirname(HERE)

FXC_OK = 0
FXC_ERR_INVALID = -1
FXC_ERR_CUDA = -2
FXC_ERR_NOMEM = -3
FXC_ERR_UNSUPPORTED = -4
FXC_ERR_NODEVICE = -5
FXC_ERR_TIMEOUT = -6

FXC_X_PLAIN_FP32 = 0
FXC_X_TC_FP16 = 1
FXC_X_TC_FP8 = 2

FXC_F_AUTO = 0
FXC_F_FFT32 = 1
FXC_F_TC16 = 2
FXC_F_TC32 = 3


class FxcConfig(C.Structure):
    """Mirror of ``fxc_config`` (include/fxcorr.h)."""
    _fields_ = [
        ("nant", C.c_int), ("npol", C.c_int), ("nchan", C.c_int), ("nbit", C.c_int),
        ("iscomplex", C.c_int), ("numffts", C.c_int), ("nsubband", C.c_int), ("xmode", C.c_int),
        ("lo", C.c_double), ("bw", C.c_double), ("sb_spacing", C.c_double), ("chunk_ffts", C.c_int),
        ("window_ffts", C.c_int), ("fstage", C.c_int),
    ]


class FxcError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = _lib().fxc_strerror(status).decode() if _LIB is not None else str(status)
        cuda = _lib().fxc_last_cuda_error() if _LIB is not None else 0
        dev = _lib().fxc_last_device_error() if _LIB is not None else 0
        super().__init__(f"{what}: {msg} (status {status}, cuda error {cuda}, device code {dev})")


_LIB = None

_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)
_FP = C.POINTER(C.c_float)

# name -> (restype, argtypes); every entry point of include/fxcorr.h
SIGNATURES = {
    "fxc_config_default": (None, [C.POINTER(FxcConfig)]),
    "fxc_subint_bytes": (C.c_size_t, [C.POINTER(FxcConfig)]),
    "fxc_num_baselines": (_I, [C.POINTER(FxcConfig)]),
    "fxc_vis_count": (C.c_size_t, [C.POINTER(FxcConfig)]),
    "fxc_create": (_I, [C.POINTER(FxcConfig), C.POINTER(_P)]),
    "fxc_destroy": (None, [_P]),
    "fxc_reset": (_I, [_P]),
    "fxc_process_host": (_I, [_P, C.POINTER(_P), _DP, _DP, _I, _I]),
    "fxc_process_device": (_I, [_P, _P, C.c_size_t, _DP, _DP, _I, _I]),
    "fxc_upload_input": (_I, [_P, C.POINTER(_P)]),
    "fxc_process_device_window": (_I, [_P, _P, C.c_size_t, C.POINTER(C.c_longlong), C.c_size_t, _DP, _DP, _I, _I]),
    "fxc_process_host_window": (_I, [_P, C.POINTER(_P), _DP, _DP, _I, _I]),
    "fxc_device_input": (_I, [_P, C.POINTER(_P), C.POINTER(C.c_size_t)]),
    "fxc_get_visibilities": (_I, [_P, _FP, _IP, _I]),
    "fxc_get_visibilities_device": (_I, [_P, _P, _I]),
    "fxc_get_amp_phase": (_I, [_P, _FP, _I]),
    "fxc_set_stream": (_I, [_P, _P]),
    "fxc_synchronize": (_I, [_P]),
    "fxc_host_alloc": (_I, [C.POINTER(_P), C.c_size_t]),
    "fxc_host_free": (_I, [_P]),
    "fxc_compat_last_error": (_I, []),
    "fxc_correlate_noalloc":(_I, [C.POINTER(FxcConfig), _P, C.c_size_t, _DP, _DP, _I, _I, _P, _P, _I, _P]),
    "fxc_set_plan": (_I, [_P, _I, _I]),
    "fxc_get_plan": (_I, [_P, _IP, _IP]),
    "fxc_autotune": (_I, [_P, _I]),
    "fxc_enable_stage_timing": (_I, [_P, _I]),
    "fxc_stage_times": (_I, [_P, _DP, C.POINTER(C.c_longlong), _I]),
    "fxc_batch_create": (_I, [C.POINTER(FxcConfig), _I, C.POINTER(_P)]),
    "fxc_batch_destroy": (None, [_P]),
    "fxc_batch_upload": (_I, [_P, _I, C.POINTER(_P)]),
    "fxc_batch_set_model": (_I, [_P, _I, _DP, _DP]),
    "fxc_batch_process": (_I, [_P]),
    "fxc_batch_reset": (_I, [_P]),
    "fxc_batch_get_visibilities": (_I, [_P, _I, _FP, _IP, _I]),
    "fxc_batch_autotune": (_I, [_P, _I]),
    "fxc_batch_get_plan": (_I, [_P, _I, _IP, _IP]),
    "fxc_batch_set_stream": (_I, [_P, _P]),
    "fxc_batch_synchronize": (_I, [_P]),
    "fxc_batch_use_graph": (_I, [_P, _I]),
    "fxc_batch_launch_count": (_I, [_P]),
    "fxc_strerror": (C.c_char_p, [_I]),
    "fxc_last_cuda_error": (_I, []),
    "fxc_last_device_error": (_I, []),
    "fxc_debug_delay_table": (_I, [_P, _DP, _DP, _I, _I, _IP, _IP, _DP, _DP, _DP]),
    "fxc_debug_unpack": (_I, [_P, _DP, _DP, _I, _I, _FP]),
    "fxc_debug_spectra": (_I, [_P, _DP, _DP, _I, _I, _FP]),
    "fxc_debug_expire_wait": (_I, [_P]),
    "fxc_debug_expire_wait_tc": (_I, [_P]),
    "fxc_debug_xplain_segments": (_I, [C.c_longlong, C.c_longlong, _I, _IP, _IP]),
}


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C difx_tests_b200/csrc` "
                              "(the correlator has no CPU implementation)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def lib():
    """The loaded libfxcorr.so (raises ImportError if it was not built)."""
    return _lib()


def _check(status, what):
    if status != FXC_OK:
        raise FxcError(status, what)


def _dp(a):
    return a.ctypes.data_as(_DP)


def make_config(nant, nchan, numffts, bw, lo, npol=2, nsubband=1, sb_spacing=None, xmode=FXC_X_PLAIN_FP32,
                chunk_ffts=0, window_ffts=0, cpx=False, fstage=FXC_F_AUTO) -> FxcConfig:
    """cpx: 8-bit complex input (FFT length nchan) instead of the reference's 2-bit real;
    fstage: F-stage arithmetic (FXC_F_*)."""
    cfg = FxcConfig()
    _lib().fxc_config_default(C.byref(cfg))
    cfg.nant, cfg.npol, cfg.nchan, cfg.numffts = nant, npol, nchan, numffts
    cfg.nsubband = nsubband
    cfg.lo, cfg.bw = float(lo), float(bw)
    cfg.sb_spacing = float(bw if sb_spacing is None else sb_spacing)
    cfg.xmode = xmode
    cfg.chunk_ffts = chunk_ffts
    cfg.window_ffts = window_ffts
    cfg.fstage = fstage
    if cpx:
        cfg.nbit, cfg.iscomplex = 8, 1
    return cfg


class Correlator:
    """One correlation context on the current CUDA device (``fxc_ctx``).

    Mirrors the reference's flow (main.c:381-441): construct (init_FxKernel),
    ``process`` FFT ranges (processAntennasAndBaselinePara; calls accumulate
    like split + merge), ``visibilities(normalize=True)`` (processNormalize).
    """

    def __init__(self, cfg: FxcConfig):
        self.cfg = cfg
        self._ctx = _P()
        _check(_lib().fxc_create(C.byref(cfg), C.byref(self._ctx)), "fxc_create")
        self.nant, self.npol, self.nchan, self.nsb = cfg.nant, cfg.npol, cfg.nchan, cfg.nsubband
        self.nbl = cfg.nant * (cfg.nant - 1) // 2
        self.subint_bytes = _lib().fxc_subint_bytes(C.byref(cfg))

    def close(self):
        if self._ctx:
            _lib().fxc_destroy(self._ctx)
            self._ctx = _P()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._ctx

    def reset(self):
        _check(_lib().fxc_reset(self._ctx), "fxc_reset")

    def process(self, data, delays, fileoffsets, first_fft=0, nfft=None):
        """data: uint8 [nsubband][nant][>= subint_bytes] host array."""
        if nfft is None:
            nfft = self.cfg.numffts - first_fft
        data, ptrs = self._row_ptrs(data)
        d = np.ascontiguousarray(delays, dtype=np.float64).reshape(-1)
        o = np.ascontiguousarray(fileoffsets, dtype=np.float64)
        _check(_lib().fxc_process_host(self._ctx, ptrs, _dp(d), _dp(o), first_fft, nfft), "fxc_process_host")

    def process_device(self, d_ptr, pitch, delays, fileoffsets, first_fft=0, nfft=None):
        if nfft is None:
            nfft = self.cfg.numffts - first_fft
        d = np.ascontiguousarray(delays, dtype=np.float64).reshape(-1)
        o = np.ascontiguousarray(fileoffsets, dtype=np.float64)
        _check(_lib().fxc_process_device(self._ctx, _P(d_ptr), pitch, _dp(d), _dp(o), first_fft, nfft),
               "fxc_process_device")

    def process_window(self, data, delays, fileoffsets, first_fft, nfft):
        """Host rows of the whole subintegration; copies only the bytes of FFTs
        [first_fft, first_fft + nfft) through the double-buffered device windows."""
        data, ptrs = self._row_ptrs(data)
        d = np.ascontiguousarray(delays, dtype=np.float64).reshape(-1)
        o = np.ascontiguousarray(fileoffsets, dtype=np.float64)
        _check(_lib().fxc_process_host_window(self._ctx, ptrs, _dp(d), _dp(o), first_fft, nfft),
               "fxc_process_host_window")

    def process_device_window(self, d_ptr, pitch, base_samples, row_bytes, delays, fileoffsets, first_fft, nfft):
        """Device rows [nsb * nant] holding each antenna's samples from base_samples[ant]."""
        b = np.ascontiguousarray(base_samples, dtype=np.int64)
        d = np.ascontiguousarray(delays, dtype=np.float64).reshape(-1)
        o = np.ascontiguousarray(fileoffsets, dtype=np.float64)
        _check(_lib().fxc_process_device_window(self._ctx, _P(d_ptr), pitch,
                                                b.ctypes.data_as(C.POINTER(C.c_longlong)), row_bytes, _dp(d), _dp(o),
                                                first_fft, nfft), "fxc_process_device_window")

    def device_input(self):
        p, pitch = _P(), C.c_size_t()
        _check(_lib().fxc_device_input(self._ctx, C.byref(p), C.byref(pitch)), "fxc_device_input")
        return p.value, pitch.value

    def visibilities(self, normalize=False, out=None):
        """-> (vis complex64 [nsb][nbl + nant][npol^2][nchan], counts int32 [nbl + nant]).

        out: optional caller-owned buffer of the same number of complex64 values (any
        shape); pinned memory (fxc_host_alloc, torch pin_memory) reads back at full
        bandwidth, a fresh pageable array goes through CUDA's staging copies."""
        n = self.nsb * (self.nbl + self.nant) * self.npol ** 2 * self.nchan
        if out is None:
            out = np.empty(2 * n, dtype=np.float32)
        else:
            out = out.reshape(-1).view(np.float32)
            if out.size != 2 * n or not out.flags.c_contiguous:
                raise ValueError("out must be a contiguous buffer of the visibility size")
        counts = np.empty(self.nbl + self.nant, dtype=np.int32)
        _check(_lib().fxc_get_visibilities(self._ctx, out.ctypes.data_as(_FP), counts.ctypes.data_as(_IP),
                                           1 if normalize else 0), "fxc_get_visibilities")
        vis = out.view(np.complex64).reshape(self.nsb, self.nbl + self.nant, self.npol ** 2, self.nchan)
        return vis, counts

    def amp_phase(self, normalize=False):
        """-> (amplitude, phase) float32 [nsb][nbl + nant][npol^2][nchan] each, computed on the
        device from the visibilities (the columns the reference's vis.out prints beside re, im)."""
        n = self.nsb * (self.nbl + self.nant) * self.npol ** 2 * self.nchan
        out = np.empty(2 * n, dtype=np.float32)
        _check(_lib().fxc_get_amp_phase(self._ctx, out.ctypes.data_as(_FP), 1 if normalize else 0),
               "fxc_get_amp_phase")
        ap = out.reshape(self.nsb, self.nbl + self.nant, self.npol ** 2, self.nchan, 2)
        return ap[..., 0], ap[..., 1]

    def visibilities_device(self, d_ptr, normalize=False):
        """Visibilities into device memory at d_ptr (vis_count complex64 values, the layout of
        visibilities()); -> counts int32 [nbl + nant] (host)."""
        _check(_lib().fxc_get_visibilities_device(self._ctx, _P(d_ptr), 1 if normalize else 0),
               "fxc_get_visibilities_device")
        counts = np.empty(self.nbl + self.nant, dtype=np.int32)
        _check(_lib().fxc_get_visibilities(self._ctx, None, counts.ctypes.data_as(_IP), 0), "fxc_get_visibilities")
        return counts

    @property
    def vis_count(self):
        return self.nsb * (self.nbl + self.nant) * self.npol ** 2 * self.nchan

    def synchronize(self):
        _check(_lib().fxc_synchronize(self._ctx), "fxc_synchronize")

    def set_stream(self, stream_ptr):
        _check(_lib().fxc_set_stream(self._ctx, _P(stream_ptr)), "fxc_set_stream")

    def set_plan(self, fft_block, x_variant=0):
        _check(_lib().fxc_set_plan(self._ctx, fft_block, x_variant), "fxc_set_plan")

    def plan(self):
        tb, alt = C.c_int(), C.c_int()
        _check(_lib().fxc_get_plan(self._ctx, C.byref(tb), C.byref(alt)), "fxc_get_plan")
        return tb.value, alt.value

    def autotune(self, reps=3):
        """Pick the fastest F-stage FFT block and plain X tile variant on the current input and
        delay model (needs one earlier process call); clears the accumulators."""
        _check(_lib().fxc_autotune(self._ctx, reps), "fxc_autotune")

    def enable_stage_timing(self, on=True):
        _check(_lib().fxc_enable_stage_timing(self._ctx, 1 if on else 0), "fxc_enable_stage_timing")

    def stage_times(self, reset=True):
        """-> (ms[4], launches[4]) for stages (delay table + counts, F, X, finalise)."""
        ms = np.zeros(4, np.float64)
        n = np.zeros(4, np.int64)
        _check(_lib().fxc_stage_times(self._ctx, _dp(ms), n.ctypes.data_as(C.POINTER(C.c_longlong)),
                                      1 if reset else 0), "fxc_stage_times")
        return ms, n

    # ---- inspection
    def delay_table(self, delays, fileoffsets, first_fft, nfft):
        A = self.nant
        off = np.empty((A, nfft), np.int32)
        val = np.empty((A, nfft), np.int32)
        frac, a, b = (np.empty((A, nfft), np.float64) for _ in range(3))
        d = np.ascontiguousarray(delays, np.float64).reshape(-1)
        o = np.ascontiguousarray(fileoffsets, np.float64)
        _check(_lib().fxc_debug_delay_table(self._ctx, _dp(d), _dp(o), first_fft, nfft, off.ctypes.data_as(_IP),
                                            val.ctypes.data_as(_IP), _dp(frac), _dp(a), _dp(b)),
               "fxc_debug_delay_table")
        return dict(offset=off, valid=val.astype(bool), frac=frac, a=a, b=b)

    def _row_ptrs(self, data):
        data = np.ascontiguousarray(data, dtype=np.uint8)
        rows = [data[s, a] for s in range(self.nsb) for a in range(self.nant)]
        return data, (_P * len(rows))(*[r.ctypes.data for r in rows])

    def upload(self, data):
        """Copy host input [nsubband][nant][>= subint_bytes] into the device input buffer."""
        data, ptrs = self._row_ptrs(data)
        _check(_lib().fxc_upload_input(self._ctx, ptrs), "fxc_upload_input")
        self.synchronize()

    _upload = upload

    def unpacked(self, data, delays, fileoffsets, first_fft, nfft):
        self._upload(data)
        F = 2 * self.nchan
        out = np.empty((self.nsb, self.nant, self.npol, nfft, F), np.float32)
        d = np.ascontiguousarray(delays, np.float64).reshape(-1)
        o = np.ascontiguousarray(fileoffsets, np.float64)
        _check(_lib().fxc_debug_unpack(self._ctx, _dp(d), _dp(o), first_fft, nfft, out.ctypes.data_as(_FP)),
               "fxc_debug_unpack")
        return out

    def spectra(self, data, delays, fileoffsets, first_fft, nfft):
        self._upload(data)
        out = np.empty((self.nsb, self.nant * self.npol, nfft, 2 * self.nchan), np.float32)
        d = np.ascontiguousarray(delays, np.float64).reshape(-1)
        o = np.ascontiguousarray(fileoffsets, np.float64)
        _check(_lib().fxc_debug_spectra(self._ctx, _dp(d), _dp(o), first_fft, nfft, out.ctypes.data_as(_FP)),
               "fxc_debug_spectra")
        return out.view(np.complex64)


class Batch:
    """Many independent correlation jobs (each its own FxcConfig, plain FP32 X
    form) processed by grouped persistent launches, replayed as one CUDA graph
    after the first call (fxc_batch_* of include/fxcorr.h)."""

    def __init__(self, cfgs):
        self.cfgs = list(cfgs)
        arr = (FxcConfig * len(self.cfgs))(*self.cfgs)
        self._b = _P()
        _check(_lib().fxc_batch_create(arr, len(self.cfgs), C.byref(self._b)), "fxc_batch_create")

    def close(self):
        if self._b:
            _lib().fxc_batch_destroy(self._b)
            self._b = _P()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, job, data):
        cfg = self.cfgs[job]
        data = np.ascontiguousarray(data, dtype=np.uint8)
        rows = [data[s, a] for s in range(cfg.nsubband) for a in range(cfg.nant)]
        ptrs = (_P * len(rows))(*[r.ctypes.data for r in rows])
        _check(_lib().fxc_batch_upload(self._b, job, ptrs), "fxc_batch_upload")

    def set_model(self, job, delays, fileoffsets):
        d = np.ascontiguousarray(delays, np.float64).reshape(-1)
        o = np.ascontiguousarray(fileoffsets, np.float64)
        _check(_lib().fxc_batch_set_model(self._b, job, _dp(d), _dp(o)), "fxc_batch_set_model")

    def process(self):
        _check(_lib().fxc_batch_process(self._b), "fxc_batch_process")

    def reset(self):
        _check(_lib().fxc_batch_reset(self._b), "fxc_batch_reset")

    def synchronize(self):
        _check(_lib().fxc_batch_synchronize(self._b), "fxc_batch_synchronize")

    def set_stream(self, stream_ptr):
        _check(_lib().fxc_batch_set_stream(self._b, _P(stream_ptr)), "fxc_batch_set_stream")

    def use_graph(self, on=True):
        _check(_lib().fxc_batch_use_graph(self._b, 1 if on else 0), "fxc_batch_use_graph")

    def autotune(self, reps=3):
        _check(_lib().fxc_batch_autotune(self._b, reps), "fxc_batch_autotune")

    def launch_count(self):
        n = _lib().fxc_batch_launch_count(self._b)
        if n < 0:
            raise FxcError(n, "fxc_batch_launch_count")
        return n

    def plan(self, job):
        tb, alt = C.c_int(), C.c_int()
        _check(_lib().fxc_batch_get_plan(self._b, job, C.byref(tb), C.byref(alt)), "fxc_batch_get_plan")
        return tb.value, alt.value

    def visibilities(self, job, normalize=False):
        cfg = self.cfgs[job]
        nbl = cfg.nant * (cfg.nant - 1) // 2
        n = cfg.nsubband * (nbl + cfg.nant) * cfg.npol ** 2 * cfg.nchan
        out = np.empty(2 * n, dtype=np.float32)
        counts = np.empty(nbl + cfg.nant, dtype=np.int32)
        _check(_lib().fxc_batch_get_visibilities(self._b, job, out.ctypes.data_as(_FP), counts.ctypes.data_as(_IP),
                                                 1 if normalize else 0), "fxc_batch_get_visibilities")
        vis = out.view(np.complex64).reshape(cfg.nsubband, nbl + cfg.nant, cfg.npol ** 2, cfg.nchan)
        return vis, counts
