"""Seeded synthetic 2-bit baseband data in the reference's file format.

Stands in for the reference's missing sample file (every antenna line of its
.conf files points at ``aa.bin``).  Model, per antenna j and polarisation p:

    x_j(t) = sqrt(rho) * s_p(t + d_j(t)) + sqrt(1 - rho) * n_jp(t),   all N(0, 1)

with a common band-limited signal s_p (independent per polarisation), station
noise n_jp, and d_j(t) = tau_j(t) - o_j the delay relative to the file start.
The delayed copy is synthesised in the frequency domain in float64 per block:
the component at baseband frequency f carries exp(+2 pi i f d_j) and the LO
phase exp(+2 pi i LO tau_j), so the correlator's integer shift, fringe rotation
and fractional-sample correction bring the antennas back into phase.

tau_j(t) = a0 + a1 t + a2 t^2 (t in seconds) is written to the .conf delay
columns as (quad, lin, const) = (a2 T^2, a1 T, a0) with T = one FFT in seconds,
because the reference evaluates the polynomial with t in FFT units
(kernel.c:378-380).  The file offset o_j is a0.

Quantisation: thresholds at +-0.98 sigma -> codes 0..3 -> levels
{-3.3359, -1, +1, +3.3359}, packed in the reference's bit order
(npol=2: kernel.c:397-426; npol=1: 4 consecutive samples per byte, LSB first).
"""
from __future__ import annotations

import dataclasses

import numpy as np

THRESH = 0.98


@dataclasses.dataclass
class Job:
    """One correlation job (one subintegration of nsubband independent subbands)."""
    nant: int
    npol: int
    nchan: int
    numffts: int
    bw: float
    lo: float
    nsubband: int
    delays: np.ndarray        # [nant][3] (quad, lin, const)
    fileoffsets: np.ndarray   # [nant] seconds
    data: np.ndarray | None   # [nsubband][nant][subintbytes] uint8 (None if generated elsewhere)
    sb_lo: np.ndarray         # [nsubband] LO (sky frequency) per subband, Hz

    @property
    def fftchannels(self) -> int:
        return 2 * self.nchan

    @property
    def subintbytes(self) -> int:
        return subint_bytes(self.nchan, self.numffts, self.npol)

    @property
    def input_samples(self) -> int:
        """Real 2-bit samples correlated: antennas x pols x subbands x FFTs x F."""
        return self.nant * self.npol * self.nsubband * self.numffts * self.fftchannels


def subint_bytes(nchan: int, numffts: int, npol: int, nbit: int = 2) -> int:
    """allocDataHost.c:21: nchan * 2 * (numffts + 1) * nbit / 8 * npol (real data)."""
    return nchan * 2 * (numffts + 1) * nbit // 8 * npol


def draw_delays(rng, nant, T_fft):
    """Quadratic delay model per antenna -> .conf columns and file offsets."""
    a0 = rng.uniform(-1e-3, 1e-3, nant)
    a1 = rng.uniform(-3e-6, 3e-6, nant)
    a2 = rng.uniform(-1e-10, 1e-10, nant)
    delays = np.stack([a2 * T_fft ** 2, a1 * T_fft, a0], axis=1)
    return delays, a0.copy()


def quantise_pack(x: np.ndarray, npol: int) -> np.ndarray:
    """x: float [npol][nsamp] (unit variance) -> packed uint8 in the reference's bit order."""
    code = np.digitize(x, [-THRESH, 0.0, THRESH]).astype(np.uint8)  # 0..3
    if npol == 2:
        nsamp = x.shape[1]
        c = code[:, : nsamp - nsamp % 2]
        return (c[0, 0::2] | (c[1, 0::2] << 2) | (c[0, 1::2] << 4) | (c[1, 1::2] << 6)).astype(np.uint8)
    c = code[0]
    c = c[: len(c) - len(c) % 4]
    return (c[0::4] | (c[1::4] << 2) | (c[2::4] << 4) | (c[3::4] << 6)).astype(np.uint8)


def _analytic_delayed(Z, d_samples):
    """Complex analytic block whose positive-frequency spectrum Z is delayed by d samples.

    Z holds bins 0..N/2 of an N-point block; bin k (k/N cycles per sample) is
    multiplied by exp(+2 pi i k d / N), i.e. the block is advanced by d samples.
    """
    N = 2 * (Z.shape[-1] - 1)
    k = np.arange(Z.shape[-1])
    full = np.zeros(N, dtype=np.complex128)
    full[: Z.shape[-1]] = Z * np.exp(2j * np.pi * k * d_samples / N)
    return np.fft.ifft(full)


def make_job(nant=4, npol=1, nchan=256, numffts=64, bw=32e6, lo=1.4e9, rho=0.1, seed=0,
             nsubband=1, sb_spacing=None, block=8192) -> Job:
    """Generate a job with numpy (sizes up to a few hundred MB of samples).

    Per block of `block` samples the delay d_j (at the block centre) is applied
    in the frequency domain to a common analytic signal; the LO phase
    exp(+2 pi i LO tau_j(t)) is applied per sample; the real part (x sqrt 2) plus
    independent noise is quantised.
    """
    rng = np.random.default_rng(seed)
    F = 2 * nchan
    Ts = 1.0 / (2.0 * bw)
    T_fft = F * Ts
    delays, fileoffsets = draw_delays(rng, nant, T_fft)
    sbb = subint_bytes(nchan, numffts, npol)
    nsamp = sbb * 8 // (2 * npol)
    if sb_spacing is None:
        sb_spacing = bw
    sb_lo = lo + sb_spacing * np.arange(nsubband)
    data = np.zeros((nsubband, nant, sbb), dtype=np.uint8)
    nblk = -(-nsamp // block)
    a0 = delays[:, 2]
    a1 = delays[:, 1] / T_fft
    a2 = delays[:, 0] / T_fft ** 2
    t = np.arange(nblk * block) * Ts
    tau = a0[:, None] + a1[:, None] * t[None, :] + a2[:, None] * t[None, :] ** 2   # [nant][nsamp]
    for sb in range(nsubband):
        x = np.zeros((nant, npol, nblk * block))
        lophase = np.exp(2j * np.pi * np.mod(sb_lo[sb] * tau, 1.0))
        for p in range(npol):
            for bi in range(nblk):
                nb = block // 2 + 1
                Z = np.sqrt(block) * (rng.standard_normal(nb) + 1j * rng.standard_normal(nb))
                Z[0] = 0.0
                tc = (bi + 0.5) * block
                sl = slice(bi * block, (bi + 1) * block)
                for j in range(nant):
                    d = (tau[j, int(tc)] - fileoffsets[j]) / Ts
                    z = _analytic_delayed(Z, d)
                    x[j, p, sl] = np.sqrt(2.0) * np.real(z * lophase[j, sl])
        x = np.sqrt(rho) * x[:, :, :nsamp] + np.sqrt(1.0 - rho) * rng.standard_normal((nant, npol, nsamp))
        for j in range(nant):
            packed = quantise_pack(x[j], npol)
            data[sb, j, : len(packed)] = packed
    return Job(nant=nant, npol=npol, nchan=nchan, numffts=numffts, bw=bw, lo=lo,
               nsubband=nsubband, delays=delays, fileoffsets=fileoffsets, data=data,
               sb_lo=sb_lo)


def make_long_job(nant=4, nchan=1024, numffts=31250, bw=64e6, lo=1.4e9, rho=0.1, seed=0, max_shift=40) -> Job:
    """A full-length subintegration of one subband, one polarisation, cheap to generate: every
    antenna sees the common N(0, 1) signal (correlation rho) shifted by a whole number of samples,
    and the delay model is that constant shift (delay -shift_j samples, file offset 0), so the
    correlator's integer shift lines the antennas up and its fringe rotation is a constant phase
    per antenna (kernel.c:428-497 with a zero delay rate).  For tests of accumulation over tens
    of thousands of FFTs, where make_job's per-sample delay synthesis would take minutes."""
    rng = np.random.default_rng(seed)
    Ts = 1.0 / (2.0 * bw)
    shifts = rng.integers(0, max_shift, nant)
    delays = np.zeros((nant, 3))
    delays[:, 2] = -shifts * Ts
    fileoffsets = np.zeros(nant)
    sbb = subint_bytes(nchan, numffts, 1)
    nsamp = sbb * 4
    common = rng.standard_normal(nsamp + max_shift, dtype=np.float32)
    data = np.zeros((1, nant, sbb), dtype=np.uint8)
    for j in range(nant):
        # stream j at sample i holds the common signal of sample i - shift_j
        sj = common[max_shift - shifts[j]: max_shift - shifts[j] + nsamp]
        x = np.sqrt(rho) * sj + np.sqrt(1.0 - rho) * rng.standard_normal(nsamp, dtype=np.float32)
        packed = quantise_pack(x[None, :], 1)
        data[0, j, : len(packed)] = packed
    return Job(nant=nant, npol=1, nchan=nchan, numffts=numffts, bw=bw, lo=lo, nsubband=1, delays=delays,
               fileoffsets=fileoffsets, data=data, sb_lo=np.array([lo]))


def subint_bytes_c8(nchan: int, numffts: int, npol: int) -> int:
    """8-bit complex input: nchan complex samples per FFT, (numffts + 1) FFTs, an int8
    (re, im) pair per sample and polarisation."""
    return nchan * (numffts + 1) * 2 * npol


def random_job(nant=4, npol=1, nchan=256, numffts=64, bw=32e6, lo=1.4e9, seed=0, nsubband=1, cpx=False):
    """Uncorrelated uniform random bytes with the same delay model (fast, any size).
    cpx: 8-bit complex samples (FFT length nchan, sample time 1/bw) instead of 2-bit real."""
    rng = np.random.default_rng(seed)
    F = nchan if cpx else 2 * nchan
    Ts = 1.0 / bw if cpx else 1.0 / (2.0 * bw)
    delays, fileoffsets = draw_delays(rng, nant, F * Ts)
    sbb = subint_bytes_c8(nchan, numffts, npol) if cpx else subint_bytes(nchan, numffts, npol)
    data = rng.integers(0, 256, size=(nsubband, nant, sbb), dtype=np.uint8)
    return Job(nant=nant, npol=npol, nchan=nchan, numffts=numffts, bw=bw, lo=lo,
               nsubband=nsubband, delays=delays, fileoffsets=fileoffsets, data=data,
               sb_lo=lo + bw * np.arange(nsubband))


def write_conf(path, job: Job, antfiles, names=None):
    """Write a reference-format .conf (main.c:14-129 grammar)."""
    names = names or [f"A{j:02d}" for j in range(job.nant)]
    with open(path, "w") as f:
        f.write("NBIT 2\nCOMPLEX 0\n")
        f.write(f"NCHAN {job.nchan}\nLO {job.lo:.1f}\nBANDWIDTH {job.bw:.1f}\n")
        f.write(f"NUMFFTS {job.numffts}\nNPOL {job.npol}\nNANT {job.nant}\n")
        for j in range(job.nant):
            q, l, c = job.delays[j]
            f.write(f"{names[j]} {antfiles[j]} {q:.17g} {l:.17g} {c:.17g} {job.fileoffsets[j]:.17g}\n")
