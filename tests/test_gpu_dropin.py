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
