"""Drive the reference's own CPU correlator (kernel.c built against ipp_shim).

Test infrastructure only.  Loads ``oracle/_ref/libfxref.so`` (built by
``oracle/Makefile`` from the reference sources) and calls the reference's entry
points exactly the way its host does (main.c:371-441): init_FxKernel ->
processAntennasAndBaselinePara over split FFT ranges -> merge -> (optionally)
processNormalize.  The reference always treats input as dual-polarisation
interleaved (kernel.c:397-426) and needs a square channel count (kernel.c:31-35).
``hoisted=True`` selects ``oracle/_ref/libfxref_hoisted.so``: the same sources with
the per-(FFT, antenna) allocKernel call of kernel.c:727-728 moved before the FFT loop
(``oracle/hoist_allockernel.py``), the secondary CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libfxref.so")
REF_LIB_HOISTED = os.path.join(HERE, "_ref", "libfxref_hoisted.so")
REF_CLI = os.path.join(HERE, "_ref", "tests_difx")

_libs = {}


def available(hoisted=False) -> bool:
    return os.path.exists(REF_LIB_HOISTED if hoisted else REF_LIB)


def lib(hoisted=False):
    _lib = _libs.get(hoisted)
    if _lib is None:
        _lib = C.CDLL(REF_LIB_HOISTED if hoisted else REF_LIB)
        _libs[hoisted] = _lib
        ip, dp, vp = C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_void_p
        _lib.init_FxKernel.argtypes = [ip, ip, ip, dp, dp, vp, C.c_char_p, ip, dp, ip, ip, ip,
                                       vp, vp, vp, vp, ip, ip, C.c_int]
        _lib.init_FxKernel.restype = None
        _lib.processAntennasAndBaselinePara.argtypes = [ip, ip, ip, dp, dp, vp, vp, vp, vp, vp,
                                                        ip, ip, ip, ip, dp, ip, vp, ip, ip, dp,
                                                        vp, ip, C.c_int]
        _lib.processAntennasAndBaselinePara.restype = None
        _lib.merge.argtypes = [C.c_int, C.c_int, vp, ip, ip, ip, vp, ip]
        _lib.merge.restype = None
        _lib.processNormalize.argtypes = [ip, ip, vp, ip, vp]
        _lib.processNormalize.restype = None
    return _lib


def _ptr_array(n):
    return (C.c_void_p * n)()


def run_reference(data, delays, fileoffsets, nchan, numffts, bw, lo, split=1, first_fft=0,
                  nfft=None, normalise=False, hoisted=False):
    """Run kernel.c on dual-pol packed input.

    data: uint8 [nant][subintbytes]; delays [nant][3]; fileoffsets [nant].
    The FFTs processed are first_fft .. first_fft+nfft-1, divided into `split`
    equal ranges as in main.c:398-408 (numffts = total FFTs of the subint sets
    maxoffset, kernel.c:730).  Returns (vis complex64 [nbl][4][nchan], counts int [nbl]).
    """
    L = lib(hoisted)
    data = np.ascontiguousarray(data, dtype=np.uint8)
    nant = data.shape[0]
    if nfft is None:
        nfft = numffts - first_fft
    if nfft % split:
        raise ValueError("nfft must divide by split")
    nbl = nant * (nant - 1) // 2
    c_nant, c_nchan, c_nbit = C.c_int(nant), C.c_int(nchan), C.c_int(2)
    c_lo, c_bw = C.c_double(lo), C.c_double(bw)
    ts = (C.c_byte * 64)()
    tstr = C.create_string_buffer(64)
    fftch, stride, sub, fraclo, nbls = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
    sampletime = C.c_double()
    unpacked, channelised, conj = _ptr_array(split * nant), _ptr_array(split * nant), _ptr_array(split * nant)
    vis = _ptr_array(split * nbl)
    count = (C.c_int * (split * nbl))()
    L.init_FxKernel(C.byref(c_nant), C.byref(c_nchan), C.byref(c_nbit), C.byref(c_lo), C.byref(c_bw),
                    C.cast(ts, C.c_void_p), tstr, C.byref(fftch), C.byref(sampletime), C.byref(stride),
                    C.byref(sub), C.byref(fraclo), C.cast(unpacked, C.c_void_p),
                    C.cast(channelised, C.c_void_p), C.cast(conj, C.c_void_p), C.cast(vis, C.c_void_p),
                    C.byref(nbls), count, split)
    # inputs
    bufs = [np.ascontiguousarray(data[a]) for a in range(nant)]
    inp = _ptr_array(nant)
    for a in range(nant):
        inp[a] = bufs[a].ctypes.data
    drows = [np.ascontiguousarray(np.asarray(delays[a], np.float64)) for a in range(nant)]
    dptr = _ptr_array(nant)
    for a in range(nant):
        dptr[a] = drows[a].ctypes.data
    offs = np.ascontiguousarray(np.asarray(fileoffsets, np.float64))
    per = nfft // split
    iters = (C.c_int * nfft)(*range(first_fft, first_fft + nfft))
    vis_out = _ptr_array(split * nbl)
    cnt_out = (C.c_int * (split * nbl))()
    c_per = C.c_int(per)
    for i in range(split):
        L.processAntennasAndBaselinePara(
            C.byref(c_nant), C.byref(c_per), C.byref(fftch), offs.ctypes.data_as(C.POINTER(C.c_double)),
            C.byref(sampletime), C.cast(inp, C.c_void_p),
            C.c_void_p(C.addressof(unpacked) + i * nant * C.sizeof(C.c_void_p)),
            C.c_void_p(C.addressof(channelised) + i * nant * C.sizeof(C.c_void_p)),
            C.c_void_p(C.addressof(conj) + i * nant * C.sizeof(C.c_void_p)),
            C.cast(dptr, C.c_void_p), C.byref(c_nbit), C.byref(sub), C.byref(stride), C.byref(fraclo),
            C.byref(c_lo), C.byref(c_nchan),
            C.c_void_p(C.addressof(vis) + i * nbl * C.sizeof(C.c_void_p)),
            C.cast(C.addressof(count) + i * nbl * C.sizeof(C.c_int), C.POINTER(C.c_int)),
            C.cast(C.addressof(iters) + i * per * C.sizeof(C.c_int), C.POINTER(C.c_int)),
            C.byref(c_bw),
            C.c_void_p(C.addressof(vis_out) + i * nbl * C.sizeof(C.c_void_p)),
            C.cast(C.addressof(cnt_out) + i * nbl * C.sizeof(C.c_int), C.POINTER(C.c_int)), split)
    merged = _ptr_array(nbl)
    mcount = (C.c_int * nbl)()
    L.merge(split, nbl, C.cast(vis, C.c_void_p), C.byref(c_nant), C.byref(c_nchan), count,
            C.cast(merged, C.c_void_p), mcount)
    if normalise:
        normed = _ptr_array(nbl)
        L.processNormalize(C.byref(nbls), count, C.cast(vis, C.c_void_p), C.byref(c_nchan),
                           C.cast(normed, C.c_void_p))
    out = np.zeros((nbl, 4, nchan), dtype=np.complex64)
    for b in range(nbl):
        rowp = C.cast(vis[b], C.POINTER(C.c_void_p))
        for p in range(4):
            arr = np.ctypeslib.as_array(C.cast(rowp[p], C.POINTER(C.c_float)), shape=(2 * nchan,))
            out[b, p] = arr[0::2] + 1j * arr[1::2]
    counts = np.array([count[b] for b in range(nbl)], dtype=np.int64)
    return out, counts
