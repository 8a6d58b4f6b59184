"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Runs the reference CPU correlator (kernel.c compiled against the IPP stand-in,
``oracle/_ref/libfxref.so`` built by ``make -C oracle``) through its exported
functions and stores inputs and outputs as .npz files:

  delay_table.npz  stationDelayAndOffset (kernel.c:938-967, the same arithmetic as
                   kernel.c:733-756) incl. negative delays, the offset == -1 and
                   maxoffset+1 nudges and invalid FFTs
  unpack.npz       unpack / unpackReal2bit (kernel.c:388-426) for even and odd offsets
  rotators.npz     fringerotate (kernel.c:428-497) and fracSampleCorrect
                   (kernel.c:512-555) applied to all-ones vectors = the rotators
  e2e_*.npz        processAntennasAndBaselinePara + merge (main.c:371-433) on
                   seeded synthetic dual-polarisation data

Usage: python tests/golden/make_golden.py   (needs the reference sources to build
oracle/_ref; the fixtures are committed so tests do not need them).
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from difx_tests_b200 import synth  # noqa: E402
from oracle import refcall  # noqa: E402


class CF32(C.Structure):
    _fields_ = [("re", C.c_float), ("im", C.c_float)]


def _cf32_pair(n):
    """cf32** with two rows of n elements (the reference's per-antenna [2][n] arrays)."""
    rows = [(CF32 * n)() for _ in range(2)]
    pp = (C.POINTER(CF32) * 2)(*[C.cast(r, C.POINTER(CF32)) for r in rows])
    return rows, pp


def _rows_to_np(rows, n):
    return np.array([[complex(r[i].re, r[i].im) for i in range(n)] for r in rows], dtype=np.complex64)


def delay_cases():
    """Per (antenna, fft): delays [3], fileoffset, numffts, F, sampletime; chosen to
    hit ordinary, negative, truncation-sensitive, nudged and invalid cases."""
    rng = np.random.default_rng(7)
    bw = 32e6
    Ts = 1.0 / (2 * bw)
    nchan = 256
    F = 2 * nchan
    numffts = 40
    cases = []
    # ordinary quadratic delays around the file offset
    for _ in range(24):
        T = F * Ts
        a0 = rng.uniform(-1e-3, 1e-3)
        d = [rng.uniform(-1e-10, 1e-10) * T * T, rng.uniform(-3e-6, 3e-6) * T, a0]
        o = a0 + rng.uniform(-3, 3) * Ts
        cases.append((d, o))
    # offsets that land exactly on the nudges / just outside the range
    for shift in (-1.0, -0.6, -0.4, 0.0, 0.4, 0.49, 0.51, 1.0, 1.4, 2.0):
        cases.append(([0.0, 0.0, 5e-6], 5e-6 + shift * Ts))            # first FFT offset near 0 / -1
        cases.append(([0.0, 0.0, -7e-6], -7e-6 - shift * Ts))           # last FFT near maxoffset(+1)
    # large positive / negative net delays (many invalid FFTs)
    cases.append(([0.0, 3 * F * Ts, 0.0], 0.0))
    cases.append(([0.0, -3 * F * Ts, 0.0], 0.0))
    cases.append(([0.0, 0.0, 100 * F * Ts], 0.0))
    return cases, dict(bw=bw, nchan=nchan, numffts=numffts)


def make_delay_table(L):
    cases, p = delay_cases()
    F = 2 * p["nchan"]
    Ts = 1.0 / (2 * p["bw"])
    L.stationDelayAndOffset.restype = None
    L.stationDelayAndOffset.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int),
                                        C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                        C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int]
    nant = len(cases)
    nf = p["numffts"]
    delays = np.array([c[0] for c in cases], np.float64)
    offs = np.array([c[1] for c in cases], np.float64)
    off = np.full((nant, nf), -999999, np.int64)
    valid = np.zeros((nant, nf), np.int64)
    frac = np.zeros((nant, nf))
    a = np.zeros((nant, nf))
    b = np.zeros((nant, nf))
    for j in range(nant):
        row = (C.c_double * 3)(*delays[j])
        dptr = (C.c_void_p * 1)(C.cast(row, C.c_void_p))
        fo = (C.c_double * 1)(offs[j])
        for k in range(nf):
            it = C.c_int(k)
            av = C.c_int(-1)
            ov = C.c_int(0)
            fr, da, db = C.c_double(0), C.c_double(0), C.c_double(0)
            st, fc = C.c_double(Ts), C.c_int(F)
            L.stationDelayAndOffset(C.cast(dptr, C.c_void_p), C.byref(it), fo, C.byref(av), C.byref(ov),
                                    C.byref(fr), C.byref(da), C.byref(db), C.byref(st), C.byref(fc), nf)
            valid[j, k] = av.value
            a[j, k], b[j, k] = da.value, db.value
            if av.value:
                off[j, k] = ov.value
                frac[j, k] = fr.value
    np.savez_compressed(os.path.join(HERE, "delay_table.npz"), delays=delays, fileoffsets=offs, bw=p["bw"],
                        nchan=p["nchan"], numffts=nf, offset=off, valid=valid, frac=frac, a=a, b=b)
    return int(valid.sum()), valid.size


def make_unpack(L):
    L.initLUT2bitReal.restype = None
    L.initLUT2bitReal()
    L.unpack.restype = None
    L.unpack.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
    rng = np.random.default_rng(11)
    nchan = 256
    F = 2 * nchan
    data = rng.integers(0, 256, size=4096, dtype=np.uint8)
    data[:256] = np.arange(256, dtype=np.uint8)  # every byte value
    offsets = np.array([0, 1, 2, 3, 5, 511, 512, 513, 1000, 1001, 2047, 4 * F + 7], np.int64)
    out = np.zeros((len(offsets), 2, F), np.float32)
    buf = np.ascontiguousarray(data)
    for i, o in enumerate(offsets):
        rows, pp = _cf32_pair(F)
        L.unpack(buf.ctypes.data, C.cast(pp, C.c_void_p), int(o), 2, F)
        out[i] = _rows_to_np(rows, F).real
    np.savez_compressed(os.path.join(HERE, "unpack.npz"), data=data, offsets=offsets, nchan=nchan, unpacked=out)


def make_rotators(L):
    L.allocKernel.restype = None
    L.allocKernel.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 4 + [C.POINTER(C.c_double)] * 2
    L.fringerotate.restype = None
    L.fringerotate.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double,
                               C.c_int, C.c_double]
    L.fracSampleCorrect.restype = None
    L.fracSampleCorrect.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_int]
    rng = np.random.default_rng(13)
    out = {}
    for nchan in (256, 1024):
        F = 2 * nchan
        stride = int(round(np.sqrt(nchan)))
        bw = 32e6 if nchan == 256 else 64e6
        Ts = 1.0 / (2 * bw)
        params = []
        for lo in (1.4e9, 1.65e9, 1.4e9 + 0.37):  # last one has a fractional LO (kernel.c:39)
            for _ in range(3):
                a = rng.uniform(-3e-6, 3e-6) * F * Ts
                b = rng.uniform(-1e-3, 1e-3) + (1.0 if rng.random() < 0.3 else 0.0)
                frac = rng.uniform(-0.5, 0.5) * Ts
                params.append((lo, a, b, frac))
        fr = np.zeros((len(params), F), np.complex64)
        fc = np.zeros((len(params), nchan), np.complex64)
        for i, (lo, a, b, frac) in enumerate(params):
            kern = (C.c_byte * 512)()
            s_sub, s_str, s_f, s_c = C.c_int(2 * stride), C.c_int(stride), C.c_int(F), C.c_int(nchan)
            ts, cbw = C.c_double(Ts), C.c_double(bw)
            L.allocKernel(C.cast(kern, C.c_void_p), C.byref(s_sub), C.byref(s_str), C.byref(s_f), C.byref(s_c),
                          C.byref(ts), C.byref(cbw))
            rows, pp = _cf32_pair(F)
            for r in rows:
                for n in range(F):
                    r[n].re, r[n].im = 1.0, 0.0
            fraclo = 1.0 if (lo - int(lo)) > 1e-11 else 0.0
            L.fringerotate(C.cast(kern, C.c_void_p), C.cast(pp, C.c_void_p), a, b, 2 * stride, stride, lo, F, fraclo)
            fr[i] = _rows_to_np(rows, F)[0]
            rows2, pp2 = _cf32_pair(F)
            for r in rows2:
                for n in range(F):
                    r[n].re, r[n].im = 1.0, 0.0
            L.fracSampleCorrect(C.cast(kern, C.c_void_p), C.cast(pp2, C.c_void_p), frac, stride, nchan)
            fc[i] = _rows_to_np(rows2, nchan)[0][:nchan]
        p = np.array(params)
        out[f"fringe_{nchan}"] = fr
        out[f"frac_{nchan}"] = fc
        out[f"params_{nchan}"] = p
        out[f"bw_{nchan}"] = bw
    np.savez_compressed(os.path.join(HERE, "rotators.npz"), **out)


def make_e2e():
    cases = {
        "e2e_c256": dict(nant=4, nchan=256, numffts=48, bw=32e6, lo=1.4e9, rho=0.1, seed=101, split=1),
        "e2e_c1024_split2": dict(nant=3, nchan=1024, numffts=16, bw=64e6, lo=1.65e9, rho=0.05, seed=102, split=2),
        "e2e_c256_fraclo": dict(nant=5, nchan=256, numffts=24, bw=32e6, lo=1.4e9 + 0.25, rho=0.2, seed=103, split=1),
    }
    for name, c in cases.items():
        job = synth.make_job(nant=c["nant"], npol=2, nchan=c["nchan"], numffts=c["numffts"], bw=c["bw"],
                             lo=c["lo"], rho=c["rho"], seed=c["seed"])
        if name == "e2e_c256":
            # antenna 3 drifts out of range: first FFTs invalid (kernel.c:752-755)
            job.delays[3, 1] = 2.5 * 2 * c["nchan"] / (2 * c["bw"])
        vis, counts = refcall.run_reference(job.data[0], job.delays, job.fileoffsets, c["nchan"], c["numffts"],
                                            c["bw"], c["lo"], split=c["split"])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), data=job.data[0], delays=job.delays,
                            fileoffsets=job.fileoffsets, nchan=c["nchan"], numffts=c["numffts"], bw=c["bw"],
                            lo=c["lo"], split=c["split"], vis=vis, counts=counts)


def main():
    if not refcall.available():
        raise SystemExit("oracle/_ref/libfxref.so missing: run `make -C oracle` with the reference sources present")
    L = refcall.lib()
    nv, nt = make_delay_table(L)
    print(f"delay_table: {nv}/{nt} valid entries")
    make_unpack(L)
    make_rotators(L)
    make_e2e()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
