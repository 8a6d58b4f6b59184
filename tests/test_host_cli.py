"""CPU tests of the command-line host's configuration and I/O error paths (no
correlation is attempted: every case fails before the GPU is used)."""
import os
import subprocess

import numpy as np
import pytest

from difx_tests_b200 import synth

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FX_CLI = os.path.join(REPO, "difx_tests_b200", "lib", "fxcorr_main")

pytestmark = pytest.mark.skipif(not os.path.exists(FX_CLI), reason="fxcorr_main not built")


def run(tmp, *args):
    return subprocess.run([FX_CLI, *args], cwd=tmp, capture_output=True, text=True, timeout=60)


def test_missing_config(tmp_path):
    r = run(tmp_path, "nope.conf")
    assert r.returncode == 1 and "nope.conf" in r.stderr


def test_insufficient_antenna_line(tmp_path):
    (tmp_path / "bad.conf").write_text("NCHAN 256\nLO 1.4e9\nBANDWIDTH 32e6\nNUMFFTS 8\nNANT 2\nAa a.bin 0 0 0\n")
    r = run(tmp_path, "bad.conf")
    assert r.returncode == 1 and "insufficient data for antenna" in r.stderr


def test_unknown_keyword_is_reported_not_fatal_and_missing_file_is(tmp_path):
    job = synth.random_job(nant=2, npol=2, nchan=256, numffts=8, seed=1)
    synth.write_conf(tmp_path / "t.conf", job, ["x0.bin", "x1.bin"])
    with open(tmp_path / "t.conf", "a") as f:
        f.write("FUTUREKEY 3\n")
    r = run(tmp_path, "t.conf")
    assert "Unknown keyword \"FUTUREKEY\"" in r.stderr
    assert r.returncode == 1 and "x0.bin" in r.stderr


def test_short_file_is_an_error(tmp_path):
    job = synth.random_job(nant=2, npol=2, nchan=256, numffts=8, seed=2)
    synth.write_conf(tmp_path / "t.conf", job, ["x0.bin", "x1.bin"])
    job.data[0, 0].tofile(tmp_path / "x0.bin")
    job.data[0, 1][:100].tofile(tmp_path / "x1.bin")
    r = run(tmp_path, "t.conf")
    assert r.returncode == 1 and "Problem reading data" in r.stderr


def test_usage(tmp_path):
    r = run(tmp_path, "-q")
    assert r.returncode == 1 and "usage" in r.stderr


def test_subband_file_pattern_needs_one_int_conversion(tmp_path):
    job = synth.random_job(nant=2, npol=2, nchan=256, numffts=8, seed=3)
    synth.write_conf(tmp_path / "t.conf", job, ["x0.bin", "x%s.bin"])
    with open(tmp_path / "t.conf", "a") as f:
        f.write("NSUBBAND 2\n")
    r = run(tmp_path, "t.conf")
    assert r.returncode == 1 and "needs one %d" in r.stderr


def test_missing_subband_stream_is_an_error(tmp_path):
    job = synth.random_job(nant=2, npol=2, nchan=256, numffts=8, seed=4)
    synth.write_conf(tmp_path / "t.conf", job, ["x0_%d.bin", "x1_%d.bin"])
    with open(tmp_path / "t.conf", "a") as f:
        f.write("NSUBBAND 2\nNSUBINT 2\n")
    for a in range(2):
        job.data[0, a].tofile(tmp_path / f"x{a}_0.bin")
    r = run(tmp_path, "t.conf", "-s", "3")
    assert r.returncode == 1 and "x0_1.bin" in r.stderr
