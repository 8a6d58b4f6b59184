"""Drop-in check: the reference's own main.c, linked against libfxcorr.so instead
of kernel.c, and this library's fxcorr_main, both produce the vis.out the
reference CLI (kernel.c + IPP stand-in) writes for the same .conf and files."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from difx_tests_b200 import synth

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_CLI = os.path.join(REPO, "oracle", "_ref", "tests_difx")
DROPIN_CLI = os.path.join(REPO, "oracle", "_ref", "tests_difx_b200")
FX_CLI = os.path.join(REPO, "difx_tests_b200", "lib", "fxcorr_main")


def read_visout(path):
    rows = np.loadtxt(path)
    return rows  # [nchan][2 + nbl*4*4]


def make_case(tmp, nant=4, nchan=256, numffts=64, seed=8):
    job = synth.make_job(nant=nant, npol=2, nchan=nchan, numffts=numffts, bw=32e6, lo=1.65e9, rho=0.1, seed=seed)
    files = []
    for a in range(nant):
        name = f"a{a}.bin"
        job.data[0, a].tofile(os.path.join(tmp, name))
        files.append(name)
    synth.write_conf(os.path.join(tmp, "test.conf"), job, files)
    return job


def run_in(tmp, exe, subdir, args=()):
    d = os.path.join(tmp, subdir)
    shutil.copytree(tmp, d, ignore=shutil.ignore_patterns("ref", "dropin", "fx"))
    r = subprocess.run([exe, *args], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return read_visout(os.path.join(d, "vis.out"))


def compare(got, ref, nbl):
    assert got.shape == ref.shape
    np.testing.assert_allclose(got[:, :2], ref[:, :2], atol=1e-6)
    cols = ref[:, 2:].reshape(ref.shape[0], nbl * 4, 4)     # re, im, amp, phase per (baseline, product)
    gcols = got[:, 2:].reshape(got.shape[0], nbl * 4, 4)
    for k in range(nbl * 4):
        ref_c = cols[:, k, 0] + 1j * cols[:, k, 1]
        got_c = gcols[:, k, 0] + 1j * gcols[:, k, 1]
        scale = np.abs(ref_c).max()
        # 1e-5 relative, plus the text format's 6-decimal quantisation
        assert np.abs(got_c - ref_c).max() <= 1e-5 * scale + 2e-6, k


@pytest.mark.skipif(not (os.path.exists(REF_CLI) and os.path.exists(DROPIN_CLI)),
                    reason="reference CLI builds not present")
def test_reference_main_linked_to_libfxcorr_matches_reference(tmp_path):
    tmp = str(tmp_path)
    make_case(tmp)
    ref = run_in(tmp, REF_CLI, "ref")
    got = run_in(tmp, DROPIN_CLI, "dropin")
    compare(got, ref, nbl=6)


@pytest.mark.skipif(not os.path.exists(REF_CLI), reason="reference CLI build not present")
def test_fxcorr_main_matches_reference_cli(tmp_path):
    tmp = str(tmp_path)
    make_case(tmp, nant=5, nchan=1024, numffts=24, seed=9)
    ref = run_in(tmp, REF_CLI, "ref")
    got = run_in(tmp, FX_CLI, "fx", args=("test.conf",))
    compare(got, ref, nbl=10)


def read_visbin(path, nrec):
    """The -b dump: per subintegration int32 {nsubband, nbl+nant, npol*npol, nchan}, int32 counts,
    complex64 visibilities."""
    raw = open(path, "rb").read()
    out, pos = [], 0
    for _ in range(nrec):
        nsb, nrow, np2, nchan = np.frombuffer(raw, np.int32, 4, pos)
        pos += 16
        counts = np.frombuffer(raw, np.int32, nrow, pos)
        pos += 4 * nrow
        n = nsb * nrow * np2 * nchan
        vis = np.frombuffer(raw, np.complex64, n, pos).reshape(nsb, nrow, np2, nchan)
        pos += 8 * n
        out.append((counts, vis))
    assert pos == len(raw)
    return out


@pytest.mark.parametrize("xmode", ["plain", "tc"])
def test_fxcorr_main_streams_subintegrations_of_several_subbands(tmp_path, xmode):
    """NSUBINT successive subintegrations of NSUBBAND per-antenna streams: subintegration s is
    FFTs s*NUMFFTS.. of each stream with the delay polynomial shifted to its first FFT, and must
    equal a one-subintegration correlation of that byte range with the shifted polynomial."""
    import dataclasses

    import difx_tests_b200 as fx

    nsub, nsb, numffts, nchan, nant = 3, 2, 40, 256, 4
    big = synth.random_job(nant=nant, npol=2, nchan=nchan, numffts=nsub * numffts, nsubband=nsb, seed=21)
    job = dataclasses.replace(big, numffts=numffts)
    names = []
    for a in range(nant):
        for sb in range(nsb):
            big.data[sb, a].tofile(tmp_path / f"ant{a}_sb{sb}.bin")
        names.append(f"ant{a}_sb%d.bin")
    synth.write_conf(tmp_path / "s.conf", job, names)
    with open(tmp_path / "s.conf", "a") as f:
        f.write(f"NSUBBAND {nsb}\nNSUBINT {nsub}\n")
    r = subprocess.run([FX_CLI, "s.conf", "-x", xmode, "-b", "vis.bin"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    recs = read_visbin(tmp_path / "vis.bin", nsub)
    for s in range(nsub):
        for sb in range(nsb):
            assert os.path.exists(tmp_path / f"vis.out.{s}.sb{sb}")

    F = 2 * nchan
    stride = numffts * F * 2 * 2 // 8                 # NUMFFTS FFTs of 2-bit, 2-pol samples
    sbb = synth.subint_bytes(nchan, numffts, 2)
    xm = fx.FXC_X_PLAIN_FP32 if xmode == "plain" else fx.FXC_X_TC_FP16
    cfg = fx.make_config(nant, nchan, numffts, job.bw, job.lo, npol=2, nsubband=nsb, xmode=xm)
    for s in range(nsub):
        k0 = float(s * numffts)
        d = np.array(job.delays, np.float64).copy()
        if s:
            for a in range(nant):
                q, l, c0 = job.delays[a]
                d[a] = (q, l + 2.0 * q * k0, c0 + l * k0 + q * k0 * k0)
        with fx.Correlator(cfg) as c:
            c.process(np.ascontiguousarray(big.data[:, :, s * stride:s * stride + sbb]), d, job.fileoffsets)
            vis, counts = c.visibilities(normalize=True)
        got_counts, got = recs[s]
        np.testing.assert_array_equal(got_counts, counts)
        want = np.asarray(vis).reshape(got.shape)
        scale = np.abs(want).max()
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-6 * scale)
