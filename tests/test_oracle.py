"""CPU tests: the FP64 oracle against the reference's own outputs.

Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from the
reference kernel.c built against the IPP stand-in) pin the oracle everywhere;
when oracle/_ref is present the oracle is also compared with the reference live
on fresh seeded inputs.
"""
import os

import numpy as np
import pytest

from difx_tests_b200 import synth
from oracle import fxoracle as fo
from oracle import refcall

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not refcall.available(), reason="oracle/_ref (reference build) not present")


def test_lut_levels():
    lut = fo.lut2bit()
    assert lut.dtype == np.float32
    assert lut[0b11100100].tolist() == [np.float32(-3.3359), -1.0, 1.0, np.float32(3.3359)]
    assert set(np.unique(lut).tolist()) == set(fo.LEVELS.tolist())


def test_delay_table_bit_exact_vs_golden(golden):
    g = golden("delay_table")
    nf = int(g["numffts"])
    tab = fo.delay_table(g["delays"], g["fileoffsets"], float(g["bw"]), int(g["nchan"]), np.arange(nf), nf)
    np.testing.assert_array_equal(tab["valid"], g["valid"].astype(bool))
    v = tab["valid"]
    np.testing.assert_array_equal(tab["offset"][v], g["offset"][v])
    # bit-exact FP64: compare the raw bit patterns
    assert np.array_equal(tab["frac"][v].view(np.int64), g["frac"][v].view(np.int64))
    assert np.array_equal(tab["a"].view(np.int64), g["a"].view(np.int64))
    assert np.array_equal(tab["b"].view(np.int64), g["b"].view(np.int64))


def test_delay_table_covers_edge_cases(golden):
    g = golden("delay_table")
    nf = int(g["numffts"])
    F = 2 * int(g["nchan"])
    Ts = 1.0 / (2 * float(g["bw"]))
    tab = fo.delay_table(g["delays"], g["fileoffsets"], float(g["bw"]), int(g["nchan"]), np.arange(nf), nf)
    v = tab["valid"]
    assert (~v).any(), "no invalid FFTs exercised"
    # a nudge moves the fractional delay outside the unnudged range [-Ts/2, Ts/2]
    assert (np.abs(tab["frac"][v]) > 0.5 * Ts * (1 + 1e-9)).any(), "no nudged offsets exercised"
    assert (tab["offset"][v] == 0).any() and (tab["offset"][v] == (nf - 1) * F).any()


def test_unpack_bit_exact_vs_golden(golden):
    g = golden("unpack")
    F = 2 * int(g["nchan"])
    got = fo.unpack(g["data"], g["offsets"], F, 2)        # [P][n][F]
    np.testing.assert_array_equal(got.transpose(1, 0, 2), g["unpacked"])


def test_rotators_vs_golden(golden):
    g = golden("rotators")
    for nchan in (256, 1024):
        params = g[f"params_{nchan}"]
        bw = float(g[f"bw_{nchan}"])
        for i, (lo, a, b, frac) in enumerate(params):
            fr = fo.fringe_rotator(a, b, lo, nchan)
            np.testing.assert_allclose(fr, g[f"fringe_{nchan}"][i], rtol=0, atol=2e-6)
            fc = fo.frac_rotator(frac, bw, nchan)
            np.testing.assert_allclose(fc, g[f"frac_{nchan}"][i], rtol=0, atol=2e-6)


@pytest.mark.parametrize("name", ["e2e_c256", "e2e_c1024_split2", "e2e_c256_fraclo"])
def test_end_to_end_vs_golden(golden, name):
    g = golden(name)
    nchan, numffts = int(g["nchan"]), int(g["numffts"])
    vis, counts = fo.correlate(g["data"], g["delays"], g["fileoffsets"], float(g["bw"]), float(g["lo"]), nchan, 2,
                               numffts=numffts)
    nbl = len(g["counts"])
    np.testing.assert_array_equal(counts[:nbl], g["counts"])
    mx, rms = fo.vis_error(g["vis"], vis[:nbl])
    assert mx.max() < 1e-5, mx.max()
    assert rms.max() < 1e-5, rms.max()


@needs_ref
@pytest.mark.parametrize("nchan,numffts,split", [(256, 32, 1), (256, 40, 4), (1024, 12, 3)])
def test_end_to_end_vs_reference_live(nchan, numffts, split):
    job = synth.make_job(nant=4, npol=2, nchan=nchan, numffts=numffts, bw=32e6, lo=1.4e9, rho=0.1, seed=nchan + split)
    vr, cr = refcall.run_reference(job.data[0], job.delays, job.fileoffsets, nchan, numffts, 32e6, 1.4e9, split=split)
    vo, co = fo.correlate(job.data[0], job.delays, job.fileoffsets, 32e6, 1.4e9, nchan, 2, numffts=numffts)
    np.testing.assert_array_equal(co[:6], cr)
    mx, _ = fo.vis_error(vr, vo[:6])
    assert mx.max() < 1e-5


@pytest.mark.skipif(not refcall.available(hoisted=True), reason="oracle/_ref (reference build) not present")
def test_hoisted_allockernel_variant_is_bit_identical():
    """The secondary CPU baseline (kernel.c with allocKernel moved out of the FFT x antenna
    loop, kernel.c:727-728) computes exactly what the as-written reference computes."""
    job = synth.make_job(nant=4, npol=2, nchan=256, numffts=24, bw=32e6, lo=1.4e9, rho=0.1, seed=77)
    va, ca = refcall.run_reference(job.data[0], job.delays, job.fileoffsets, 256, 24, 32e6, 1.4e9, split=2)
    vh, ch = refcall.run_reference(job.data[0], job.delays, job.fileoffsets, 256, 24, 32e6, 1.4e9, split=2,
                                   hoisted=True)
    np.testing.assert_array_equal(ca, ch)
    np.testing.assert_array_equal(va, vh)


def test_hoist_script_moves_exactly_the_per_iteration_alloc():
    import importlib.util
    spec = importlib.util.spec_from_file_location("hoist", os.path.join(REPO, "oracle", "hoist_allockernel.py"))
    h = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(h)
    src = ("void processAntennasAndBaselinePara(int *n) {\n    int netdelaysamples, offset;\n"
           "    for (k = 0; k < 2; k++) {\n        for (j = 0; j < 2; j++) {\n            FxKernel kernel;\n"
           "            allocKernel(&kernel, a, b);\n            use(&kernel);\n        }\n    }\n}\n"
           "\nvoid processBaselinePara(int *n) {}\n")
    out = h.hoist(src)
    assert out.count("allocKernel(&kernel") == 1
    assert out.index("allocKernel(&kernel") < out.index("for (k = 0")
    with pytest.raises(SystemExit):
        h.hoist(src.replace("allocKernel(&kernel, a, b);", ""))


def test_normalise_matches_reference_semantics():
    vis = np.ones((3, 1, 4), np.complex128) * (6 + 3j)
    counts = np.array([3, 0, 2])
    out = fo.normalise(vis, counts)
    np.testing.assert_allclose(out[0], 2 + 1j)
    np.testing.assert_allclose(out[1], 6 + 3j)  # count 0: left as is (kernel.c:350)
    np.testing.assert_allclose(out[2], 3 + 1.5j)


def test_nonsquare_geometry_and_frac_closed_form():
    for nchan in (128, 512, 2048, 4096):
        F, stride, S = fo.geometry(nchan)
        assert F == stride * S
        frac = 7.3e-9
        bw = 64e6
        r = fo.frac_rotator(frac, bw, nchan, ref_args=False)
        c = np.arange(nchan)
        np.testing.assert_allclose(r, np.exp(2j * np.pi * c * bw / nchan * frac), atol=1e-5)


def test_single_pol_unpack_order():
    # npol=1: 4 consecutive samples per byte, LSB first
    data = np.array([0b11100100, 0b00011011], np.uint8)
    got = fo.unpack(data, np.array([0, 1, 3]), 4, 1)[0]
    L = fo.LEVELS
    np.testing.assert_array_equal(got[0], [L[0], L[1], L[2], L[3]])
    np.testing.assert_array_equal(got[1], [L[1], L[2], L[3], L[3]])
    np.testing.assert_array_equal(got[2], [L[3], L[3], L[2], L[1]])


def test_generator_phases_align():
    """Synthetic data: corrected cross phases ~0 and |V_cross|/|V_auto| ~ rho x quantiser efficiency."""
    job = synth.make_job(nant=3, npol=1, nchan=256, numffts=96, bw=32e6, lo=1.4e9, rho=0.2, seed=5)
    vis, counts = fo.correlate(job.data[0], job.delays, job.fileoffsets, 32e6, 1.4e9, 256, 1, numffts=96)
    V = fo.normalise(vis, counts)
    nbl = 3
    cross = V[:nbl, 0, 8:-8].mean(axis=-1)
    auto = np.abs(V[nbl:, 0, 8:-8].mean(axis=-1)).mean()
    assert np.all(np.abs(np.angle(cross)) < 0.15)
    ratio = np.abs(cross) / auto
    assert np.all((ratio > 0.12) & (ratio < 0.22)), ratio


def test_unpack_c8_byte_layout():
    """8-bit complex: int8 (re, im) per sample and polarisation, polarisations interleaved."""
    npol, F = 2, 4
    raw = np.arange(2 * npol * 8, dtype=np.int16) - 10          # samples 0..7
    data = raw.astype(np.int8).view(np.uint8)
    x = fo.unpack_c8(data, np.array([1, 3]), F, npol)          # [pol][fft][n]
    for k, off in enumerate((1, 3)):
        for p in range(npol):
            for n in range(F):
                i = 2 * ((off + n) * npol + p)
                assert x[p, k, n] == complex(raw[i], raw[i + 1])
    assert synth.subint_bytes_c8(1024, 99, 2) == 1024 * 100 * 4


def test_complex_geometry_and_delays():
    F, stride, S = fo.geometry(1024, cpx=True)
    assert (F, stride, S) == (1024, 32, 32)
    job = synth.random_job(nant=3, npol=1, nchan=512, numffts=40, bw=64e6, seed=5, cpx=True)
    tab = fo.delay_table(job.delays, job.fileoffsets, job.bw, job.nchan, np.arange(40), 40, cpx=True)
    # offsets in complex samples (sample time 1/bw), FFT length nchan
    a, b, mean = fo.station_delay(job.delays, np.arange(40))
    n = np.trunc((mean - job.fileoffsets[:, None]) * job.bw + 0.5).astype(np.int64)
    expect = np.arange(40)[None, :] * 512 - n
    v = tab["valid"]
    np.testing.assert_array_equal(tab["offset"][v], expect[v])
