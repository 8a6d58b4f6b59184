"""FP64 CPU restatement of the reference FX correlator (test infrastructure only).

This is the oracle: tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline use it as the checker.  The product never imports it.

Each function restates one step of the reference's CPU path (``kernel.c`` of
twiG56/difx_tests) in numpy:

* integer/FP64 bookkeeping (delay polynomial, integer offset, nudges, validity,
  2-bit decode) follows the reference operation by operation, so it is
  bit-exact with ``kernel.c`` compiled by gcc on x86-64 (IEEE binary64, no FMA);
* the signal processing (fringe rotation, FFT, fractional-sample correction,
  cross-multiply-accumulate) runs in float64.  With ``ref_args=True`` the phase
  arguments are rounded to float32 exactly where ``kernel.c`` stores them as
  ``f32`` (kernel.c:463-470, 517-523), so the only differences from the
  reference are the reference's own float32 roundings.

Generalisations beyond the reference's CPU path (documented, used by the GPU
path's parity tests): single polarisation input (4 consecutive samples per
byte, LSB first), non-square channel counts, autocorrelations, several
independent subbands, and 8-bit complex input (``cpx=True``).

8-bit complex input is the reference's GPU-path format, which its CPU path
rejects (kernel.c:392-394): each time sample is an int8 (re, im) pair per
polarisation, polarisations interleaved per sample (gkernel.cu:277-296), sampled
at the bandwidth (sampletime 1/bw, main_gpu.cu:246-247) with FFT length nchan
(cfactor 1, main_gpu.cu:236-242), every FFT bin a channel.  The CPU path's own
formulas carry over with that FFT length: substride = (2/cfact)*stride
(kernel.c:16, 36) = F/stride, the rotator and fractional-sample tables
unchanged.  No reference CPU output exists for this format, so its parity rests
on these shared, pinned formulas; the unpack restates gkernel.cu's byte layout.
"""
from __future__ import annotations

import math

import numpy as np

# kernel.c:191-192 -- 4-level quantiser levels ("HiMag" = 3.3359, optimal value)
HIMAG = np.float32(3.3359)
LEVELS = np.array([-HIMAG, -1.0, 1.0, HIMAG], dtype=np.float32)
TWO_PI = 2.0 * 3.14159265358979323846  # vectordefs.h:4 (2*IPP_PI)


def lut2bit() -> np.ndarray:
    """256x4 float32 decode table, kernel.c:189-202: lut[b][i] = L[(b >> 2i) & 3]."""
    b = np.arange(256)[:, None]
    i = np.arange(4)[None, :]
    return LEVELS[(b >> (2 * i)) & 3]


def geometry(nchan: int, cpx: bool = False):
    """Derived sizes, kernel.c:13-36 generalised to any power-of-two channel count.

    Returns (fftchannels F, stride, substride S).  The reference requires nchan
    to be a perfect square (kernel.c:31-35) with stride = sqrt(nchan) and
    substride = 2*stride = F/stride.  For other powers of two the same
    factorisation F = stride * S is kept with stride = 2^floor(log2(nchan)/2).
    """
    if nchan <= 0 or nchan & (nchan - 1):
        raise ValueError("nchan must be a power of two")
    F = nchan if cpx else 2 * nchan
    stride = 1 << (int(math.log2(nchan)) // 2)
    S = F // stride
    return F, stride, S


def station_delay(delays: np.ndarray, fftindex: np.ndarray):
    """kernel.c:373-386 getStationDelay, vectorised over antennas x FFTs.

    delays: [nant][3] = (quad, lin, const) in seconds per FFT-index power.
    fftindex: [nfft] absolute FFT indices.
    Returns (a, b, meandelay), each [nant][nfft] float64.
    """
    q = delays[:, 0:1].astype(np.float64)
    l = delays[:, 1:2].astype(np.float64)
    c = delays[:, 2:3].astype(np.float64)
    k = np.asarray(fftindex, dtype=np.float64)[None, :]
    d0 = q * k * k + l * k + c
    kh = k + 0.5
    d1 = q * kh * kh + l * kh + c
    k1 = k + 1.0
    d2 = q * k1 * k1 + l * k1 + c
    a = d2 - d0
    b = d0 + (d1 - (a * 0.5 + d0)) / 3.0
    mean = a * 0.5 + b
    return a, b, mean


def delay_table(delays, fileoffsets, bw, nchan, fftindex, maxoffset_ffts, cpx=False):
    """kernel.c:733-756: integer sample offset, fractional delay and validity.

    maxoffset_ffts is numffts*split of the reference (total FFTs of the
    subintegration), so maxoffset = (maxoffset_ffts - 1) * F (kernel.c:730).
    Returns dict of [nant][nfft] arrays: offset (int64), frac (float64 seconds),
    valid (bool), a, b (float64).
    """
    F = nchan if cpx else 2 * nchan
    sampletime = 1.0 / bw if cpx else 1.0 / (2.0 * bw)  # main_gpu.cu:246-247 / kernel.c:14
    a, b, mean = station_delay(np.asarray(delays, np.float64), fftindex)
    off = np.asarray(fileoffsets, np.float64)[:, None]
    nf = (mean - off) / sampletime
    n = np.trunc(nf + 0.5).astype(np.int64)  # (int)(x + 0.5): C truncation toward zero
    frac = -(nf - n) * sampletime
    k = np.asarray(fftindex, np.int64)[None, :]
    offset = k * F - n
    maxoffset = (int(maxoffset_ffts) - 1) * F
    lo_nudge = offset == -1
    offset = np.where(lo_nudge, 0, offset)
    frac = np.where(lo_nudge, frac + sampletime, frac)
    hi_nudge = offset == maxoffset + 1
    offset = np.where(hi_nudge, offset - 1, offset)
    frac = np.where(hi_nudge, frac - sampletime, frac)
    valid = (offset >= 0) & (offset <= maxoffset)
    return dict(offset=offset, frac=frac, valid=valid, a=a, b=b)


def unpack(data: np.ndarray, offsets: np.ndarray, F: int, npol: int) -> np.ndarray:
    """kernel.c:397-426 unpackReal2bit, vectorised; returns float32 [npol][nfft][F].

    npol=2 (the reference's only format): byte s//2 holds time samples s, s+1 of
    both polarisations, bits 1:0 = (t0,p0), 3:2 = (t0,p1), 5:4 = (t1,p0),
    7:6 = (t1,p1).  npol=1: byte s//4 holds 4 consecutive samples, bits 2i..2i+1.
    Sample n of an FFT is absolute sample offset+n.
    """
    s = offsets[:, None].astype(np.int64) + np.arange(F, dtype=np.int64)[None, :]
    out = np.empty((npol,) + s.shape, dtype=np.float32)
    if npol == 2:
        byte = data[s // 2].astype(np.int64)
        sh = 4 * (s % 2)
        for p in range(2):
            out[p] = LEVELS[(byte >> (sh + 2 * p)) & 3]
    elif npol == 1:
        byte = data[s // 4].astype(np.int64)
        out[0] = LEVELS[(byte >> (2 * (s % 4))) & 3]
    else:
        raise ValueError("npol must be 1 or 2")
    return out


def unpack_c8(data: np.ndarray, offsets: np.ndarray, F: int, npol: int) -> np.ndarray:
    """8-bit complex samples (gkernel.cu:277-296 byte layout): sample s of polarisation
    p is the int8 pair at bytes 2*(s*npol + p), 2*(s*npol + p) + 1; returns complex128
    [npol][nfft][F] for samples offset .. offset+F-1."""
    s = offsets[:, None].astype(np.int64) + np.arange(F, dtype=np.int64)[None, :]
    b = np.asarray(data).view(np.int8)
    out = np.empty((npol,) + s.shape, dtype=np.complex128)
    for p in range(npol):
        i = 2 * (s * npol + p)
        out[p] = b[i].astype(np.float64) + 1j * b[i + 1].astype(np.float64)
    return out


def _frac_int(x):
    """x - (int)x with C truncation (kernel.c:434-435, 465, 469)."""
    return x - np.trunc(x)


def fringe_rotator(a, b, lo, nchan, ref_args=True, cpx=False):
    """kernel.c:428-488: complex rotator for one FFT per (a, b) pair.

    a, b: float64 arrays (any shape).  Returns complex128 [..., F].
    rot[i*S + j] = sub[j] * step[i] with
      sub[j]  = exp(i*subarg[j]),  subarg[j]  = -2pi*frac(lo*(j/F*a + b'))
      step[i] = exp(i*steparg[i]), steparg[i] = -2pi*frac(lo*(i*stride/F*a))
    where b' = b - (int)b, plus lo_frac*(int)b turns when lo is fractional
    (kernel.c:455-460).  The step spacing i*stride/F (kernel.c:145) is the
    reference's formula and is kept as is.
    """
    F, stride, S = geometry(nchan, cpx)
    out_shape = np.broadcast(np.asarray(a), np.asarray(b)).shape + (F,)
    a = np.asarray(a, np.float64)[..., None]
    b = np.asarray(b, np.float64)[..., None]
    intdelay = np.trunc(b)
    b = b - intdelay
    subxoff = np.arange(S, dtype=np.float64) / float(F)
    stepxoff = (np.arange(stride, dtype=np.float64) * float(stride)) / float(F)
    subphase = (subxoff * a + b) * lo
    stepphase = (stepxoff * a) * lo
    if (lo - math.trunc(lo)) > 1e-11:  # kernel.c:39 fractionalLoFreq
        subphase = subphase + (lo - math.trunc(lo)) * intdelay
    subarg = -TWO_PI * _frac_int(subphase)
    steparg = -TWO_PI * _frac_int(stepphase)
    if ref_args:
        subarg = subarg.astype(np.float32).astype(np.float64)
        steparg = steparg.astype(np.float32).astype(np.float64)
    sub = np.exp(1j * subarg)            # [..., S]
    step = np.exp(1j * steparg)          # [..., stride]
    rot = step[..., :, None] * sub[..., None, :]   # [..., stride, S]
    return rot.reshape(out_shape)


def channel_freq_tables(bw, nchan):
    """kernel.c:162-166: float32 sub/step channel angular frequencies.

    subchannelfreqs[j]  = (f32)(2pi*j*bw/nchan),        j < stride
    stepchannelfreqs[i] = (f32)(2pi*i*stride*bw/nchan), i < nchan/stride
    """
    _, stride, _ = geometry(nchan)
    j = np.arange(stride, dtype=np.float64)
    i = np.arange(nchan // stride, dtype=np.float64)
    sub = ((TWO_PI * j * bw) / float(nchan)).astype(np.float32)
    step = ((TWO_PI * i * stride * bw) / float(nchan)).astype(np.float32)
    return sub, step


def frac_rotator(frac, bw, nchan, ref_args=True):
    """kernel.c:512-546: fractional-sample correction rotator, [..., nchan] complex128.

    rot[i*stride + j] = exp(i*f32(sub[j]*f32(frac))) * exp(i*f32(step[i]*f32(frac)))
    which equals exp(+2pi*i*c*bw*frac/nchan) up to float32 argument rounding.
    """
    _, stride, _ = geometry(nchan)
    sub, step = channel_freq_tables(bw, nchan)
    out_shape = np.shape(frac) + (nchan,)
    frac = np.asarray(frac, np.float64)[..., None]
    if ref_args:
        f32 = frac.astype(np.float32)
        subarg = (sub[None, :] * f32).astype(np.float32).astype(np.float64)
        steparg = (step[None, :] * f32).astype(np.float32).astype(np.float64)
    else:
        subarg = sub.astype(np.float64) * frac
        steparg = step.astype(np.float64) * frac
    rot = np.exp(1j * steparg)[..., :, None] * np.exp(1j * subarg)[..., None, :]
    return rot.reshape(out_shape)


def channelise(data, delays, fileoffsets, bw, lo, nchan, npol, fftindex, maxoffset_ffts,
               ref_args=True, cpx=False):
    """Per antenna: unpack -> fringe rotate -> FFT -> fractional-sample correct.

    Follows kernel.c:725-789 for every FFT in fftindex.  data: [nant][nbytes]
    uint8.  Returns (spectra complex128 [nant][npol][nfft][nchan] -- zero where
    the antenna is invalid for that FFT --, delay-table dict).
    """
    data = np.asarray(data)
    nant = data.shape[0]
    F = nchan if cpx else 2 * nchan
    tab = delay_table(delays, fileoffsets, bw, nchan, fftindex, maxoffset_ffts, cpx)
    nfft = len(fftindex)
    spec = np.zeros((nant, npol, nfft, nchan), dtype=np.complex128)
    for ant in range(nant):
        v = tab["valid"][ant]
        if not v.any():
            continue
        idx = np.nonzero(v)[0]
        if cpx:
            x = unpack_c8(data[ant], tab["offset"][ant, idx], F, npol)                 # [P][n][F]
        else:
            x = unpack(data[ant], tab["offset"][ant, idx], F, npol).astype(np.float64)  # [P][n][F]
        rot = fringe_rotator(tab["a"][ant, idx], tab["b"][ant, idx], lo, nchan, ref_args, cpx)
        X = np.fft.fft(x * rot[None], axis=-1)[..., :nchan]
        X = X * frac_rotator(tab["frac"][ant, idx], bw, nchan, ref_args)[None]
        spec[ant][:, idx, :] = X
    return spec, tab


def baseline_order(nant):
    """Cross baselines in the reference's order (kernel.c:832-852): (0,1),(0,2)..(A-2,A-1)."""
    return [(j, k) for j in range(nant - 1) for k in range(j + 1, nant)]


def correlate(data, delays, fileoffsets, bw, lo, nchan, npol, fftindex=None, numffts=None,
              maxoffset_ffts=None, ref_args=True, chunk=256, cpx=False):
    """Full per-subintegration FX correlation in float64 (kernel.c:709-854).

    Returns (vis, counts):
      vis    complex128 [nbl + nant][npol*npol][nchan]: the nbl = A(A-1)/2 cross
             baselines in reference order, then the A autocorrelations; product
             index 2*l + m (kernel.c:846) for polarisations (l, m); NOT normalised
             (the reference's accumulators before processNormalize).
      counts int64 [nbl + nant]: FFTs where both antennas were valid.
    """
    data = np.asarray(data)
    nant = data.shape[0]
    if fftindex is None:
        fftindex = np.arange(numffts)
    fftindex = np.asarray(fftindex, np.int64)
    if maxoffset_ffts is None:
        maxoffset_ffts = numffts if numffts is not None else len(fftindex)
    nsig = nant * npol
    V = np.zeros((nchan, nsig, nsig), dtype=np.complex128)
    valid_all = np.zeros((nant, len(fftindex)), dtype=bool)
    for c0 in range(0, len(fftindex), chunk):
        idx = fftindex[c0:c0 + chunk]
        spec, tab = channelise(data, delays, fileoffsets, bw, lo, nchan, npol, idx,
                               maxoffset_ffts, ref_args, cpx=cpx)
        valid_all[:, c0:c0 + len(idx)] = tab["valid"]
        X = spec.reshape(nsig, len(idx), nchan).transpose(2, 0, 1)  # [C][sig][t]
        V += X @ np.conj(X).transpose(0, 2, 1)
    bls = baseline_order(nant) + [(a, a) for a in range(nant)]
    vis = np.zeros((len(bls), npol * npol, nchan), dtype=np.complex128)
    counts = np.zeros(len(bls), dtype=np.int64)
    for bi, (j, k) in enumerate(bls):
        for l in range(npol):
            for m in range(npol):
                vis[bi, l * npol + m] = V[:, j * npol + l, k * npol + m]
        counts[bi] = int(np.count_nonzero(valid_all[j] & valid_all[k]))
    return vis, counts


def normalise(vis, counts):
    """kernel.c:348-359 processNormalize: divide each baseline by its count (skip 0)."""
    out = vis.copy()
    nz = counts > 0
    out[nz] = out[nz] / counts[nz][:, None, None]
    return out


def vis_error(test, ref):
    """Per product spectrum error metrics against a reference.

    Returns (max_rel, rms_rel) arrays shaped like test.shape[:-1]:
      max_rel = max|test - ref| / max|ref|,  rms_rel = ||test - ref||_2 / ||ref||_2.
    Spectra whose reference is identically zero report 0 if test is zero too.
    """
    d = np.abs(np.asarray(test) - np.asarray(ref))
    r = np.abs(np.asarray(ref))
    rmax = r.max(axis=-1)
    rn = np.sqrt((r ** 2).sum(axis=-1))
    dmax = d.max(axis=-1)
    dn = np.sqrt((d ** 2).sum(axis=-1))
    with np.errstate(divide="ignore", invalid="ignore"):
        max_rel = np.where(rmax > 0, dmax / np.where(rmax > 0, rmax, 1), dmax)
        rms_rel = np.where(rn > 0, dn / np.where(rn > 0, rn, 1), dn)
    return max_rel, rms_rel
