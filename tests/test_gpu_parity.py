"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Bars: integer/bit work (delay table, unpacked samples) bit-exact; FP32 spectra
and plain-form visibilities within 1e-5 relative (max|d| / max|ref| per spectrum)
of the reference kernel.c outputs (golden fixtures) and of the FP64 oracle.
"""
import numpy as np
import pytest

import difx_tests_b200 as fx
from difx_tests_b200 import synth
from oracle import fxoracle as fo
from oracle import refcall

pytestmark = pytest.mark.gpu

VIS_TOL = 1e-5       # plain FP32 form vs reference / FP64 oracle, relative to max|V| per spectrum
SPEC_TOL = 2e-5      # FP32 F stage vs FP64 oracle, relative to max|X| per spectrum


def corr_for(job, **kw):
    cfg = fx.make_config(job.nant, job.nchan, job.numffts, job.bw, job.lo, npol=job.npol, nsubband=job.nsubband,
                         sb_spacing=(job.sb_lo[1] - job.sb_lo[0]) if job.nsubband > 1 else job.bw, **kw)
    return fx.Correlator(cfg)


def oracle_vis(job, sb=0, fftindex=None):
    lo = float(job.sb_lo[sb])
    return fo.correlate(job.data[sb], job.delays, job.fileoffsets, job.bw, lo, job.nchan, job.npol,
                        fftindex=fftindex, numffts=job.numffts, maxoffset_ffts=job.numffts)


def assert_vis_close(got, ref, tol=VIS_TOL):
    mx, rms = fo.vis_error(got, ref)
    assert mx.max() < tol, f"max rel err {mx.max():.3e} (rms {rms.max():.3e})"


def test_delay_table_bit_exact_vs_reference(golden):
    g = golden("delay_table")
    nant = g["delays"].shape[0]
    nf = int(g["numffts"])
    cfg = fx.make_config(nant, int(g["nchan"]), nf, float(g["bw"]), 1.4e9, npol=1)
    with fx.Correlator(cfg) as c:
        tab = c.delay_table(g["delays"], g["fileoffsets"], 0, nf)
    np.testing.assert_array_equal(tab["valid"], g["valid"].astype(bool))
    v = tab["valid"]
    np.testing.assert_array_equal(tab["offset"][v], g["offset"][v])
    assert np.array_equal(tab["frac"][v].view(np.int64), g["frac"][v].view(np.int64))
    assert np.array_equal(tab["a"].view(np.int64), g["a"].view(np.int64))
    assert np.array_equal(tab["b"].view(np.int64), g["b"].view(np.int64))


@pytest.mark.parametrize("nchan,first", [(256, 0), (2048, 17), (4096, 5)])
def test_delay_table_bit_exact_vs_oracle(nchan, first):
    job = synth.random_job(nant=9, npol=1, nchan=nchan, numffts=300, bw=64e6, seed=nchan)
    Ts = 1.0 / (2 * job.bw)
    job.delays[2, 1] = 0.5 * 2 * nchan * Ts   # drifts half an FFT per FFT: out of range at the end
    job.fileoffsets[4] -= 50.3 * 2 * nchan * Ts   # net delay 50 FFTs: the first FFTs are invalid
    job.fileoffsets[3] += 0.6 * Ts
    nf = 200
    with corr_for(job) as c:
        tab = c.delay_table(job.delays, job.fileoffsets, first, nf)
    ref = fo.delay_table(job.delays, job.fileoffsets, job.bw, nchan, np.arange(first, first + nf), job.numffts)
    np.testing.assert_array_equal(tab["valid"], ref["valid"])
    v = ref["valid"]
    assert (~v).any()
    np.testing.assert_array_equal(tab["offset"][v], ref["offset"][v])
    assert np.array_equal(tab["frac"][v].view(np.int64), ref["frac"][v].view(np.int64))


@pytest.mark.parametrize("npol", [1, 2])
@pytest.mark.parametrize("nchan", [128, 256, 1024, 4096])
def test_unpack_bit_exact(npol, nchan):
    job = synth.random_job(nant=3, npol=npol, nchan=nchan, numffts=20, bw=32e6, seed=npol * 7 + nchan)
    job.fileoffsets[1] += 1.0 / (2 * job.bw)      # odd offsets
    job.fileoffsets[2] += 3.0 / (2 * job.bw)
    with corr_for(job) as c:
        got = c.unpacked(job.data, job.delays, job.fileoffsets, 0, job.numffts)[0]   # [ant][pol][t][F]
    tab = fo.delay_table(job.delays, job.fileoffsets, job.bw, nchan, np.arange(job.numffts), job.numffts)
    F = 2 * nchan
    for a in range(job.nant):
        v = tab["valid"][a]
        ref = fo.unpack(job.data[0, a], tab["offset"][a][v], F, npol)    # [P][n][F]
        np.testing.assert_array_equal(got[a][:, v, :], ref)
        assert np.all(got[a][:, ~v, :] == 0)


def test_unpack_matches_reference_golden(golden):
    g = golden("unpack")
    nchan = int(g["nchan"])
    F = 2 * nchan
    # drive the F stage's decoder with offsets from a constant-delay model: one antenna per golden offset
    offs = g["offsets"]
    nant = len(offs)
    bw = 32e6
    Ts = 1.0 / (2 * bw)
    numffts = 16                                   # subint_bytes = 4352 >= len(data)
    cfg = fx.make_config(nant, nchan, numffts, bw, 1.4e9, npol=2)
    delays = np.zeros((nant, 3))
    # nf = -(o + 1)  ->  n = (int)(nf + 0.5) = -o (truncation toward zero)  ->  offset(k=0) = o
    fileoffsets = np.array([(o + 1.0) * Ts for o in offs])
    data = np.zeros((1, nant, fx.lib().fxc_subint_bytes(cfg)), np.uint8)
    data[0, :, : len(g["data"])] = g["data"][None, :]
    with fx.Correlator(cfg) as c:
        got = c.unpacked(data, delays, fileoffsets, 0, 1)[0][:, :, 0, :]   # [ant][pol][F]
    np.testing.assert_array_equal(got, g["unpacked"])


@pytest.mark.parametrize("npol", [1, 2])
@pytest.mark.parametrize("nchan", [128, 256, 512, 1024, 2048, 4096])
def test_spectra_vs_fp64(npol, nchan):
    nf = 24
    job = synth.random_job(nant=2, npol=npol, nchan=nchan, numffts=nf, bw=64e6, lo=1.4e9 + 0.3, seed=nchan + npol)
    with corr_for(job) as c:
        got = c.spectra(job.data, job.delays, job.fileoffsets, 0, nf)[0]         # [sig][t][C]
    spec, tab = fo.channelise(job.data[0], job.delays, job.fileoffsets, job.bw, job.lo, nchan, npol,
                              np.arange(nf), nf)
    ref = spec.reshape(job.nant * npol, nf, nchan)
    err = np.abs(got - ref).max(axis=-1) / np.maximum(np.abs(ref).max(axis=-1), 1e-30)
    valid = np.repeat(tab["valid"], npol, axis=0)
    assert err[valid].max() < SPEC_TOL, err[valid].max()
    assert np.all(got[~valid] == 0)


@pytest.mark.parametrize("name", ["e2e_c256", "e2e_c1024_split2", "e2e_c256_fraclo"])
def test_vis_vs_reference_golden(golden, name):
    g = golden(name)
    nchan, numffts = int(g["nchan"]), int(g["numffts"])
    nant = g["data"].shape[0]
    cfg = fx.make_config(nant, nchan, numffts, float(g["bw"]), float(g["lo"]), npol=2)
    with fx.Correlator(cfg) as c:
        split = int(g["split"])
        per = numffts // split
        for i in range(split):     # the reference's split ranges, accumulated (merge)
            c.process(g["data"][None], g["delays"], g["fileoffsets"], i * per, per)
        vis, counts = c.visibilities()
    nbl = len(g["counts"])
    np.testing.assert_array_equal(counts[:nbl], g["counts"])
    assert_vis_close(vis[0, :nbl], g["vis"])


@pytest.mark.skipif(not refcall.available(), reason="oracle/_ref not present")
def test_vis_vs_reference_live():
    job = synth.make_job(nant=6, npol=2, nchan=256, numffts=64, bw=32e6, lo=1.65e9, rho=0.1, seed=21)
    vr, cr = refcall.run_reference(job.data[0], job.delays, job.fileoffsets, 256, 64, 32e6, 1.65e9)
    with corr_for(job) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    np.testing.assert_array_equal(counts[:15], cr)
    assert_vis_close(vis[0, :15], vr)


@pytest.mark.parametrize("nant,npol,nchan,nsb", [(4, 1, 256, 1), (8, 2, 512, 2), (16, 2, 2048, 1), (64, 1, 1024, 1),
                                                  (12, 1, 128, 3), (5, 2, 4096, 1)])
def test_vis_vs_fp64_oracle(nant, npol, nchan, nsb):
    numffts = 40 if nchan <= 1024 else 16
    job = synth.make_job(nant=nant, npol=npol, nchan=nchan, numffts=numffts, bw=64e6, lo=1.4e9, rho=0.1,
                         seed=nant * 100 + nchan, nsubband=nsb)
    with corr_for(job) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    for sb in range(nsb):
        ref, rc = oracle_vis(job, sb)
        np.testing.assert_array_equal(counts, rc)
        assert_vis_close(vis[sb], ref)


def test_time_shards_and_chunks_accumulate():
    job = synth.make_job(nant=5, npol=1, nchan=256, numffts=200, bw=32e6, lo=1.4e9, rho=0.1, seed=77)
    ref, rc = oracle_vis(job)
    with corr_for(job, chunk_ffts=64) as c:
        for first, n in [(0, 37), (37, 100), (137, 63)]:
            c.process(job.data, job.delays, job.fileoffsets, first, n)
        vis, counts = c.visibilities()
        np.testing.assert_array_equal(counts, rc)
        assert_vis_close(vis[0], ref)
        visn, _ = c.visibilities(normalize=True)
        assert_vis_close(visn[0], fo.normalise(ref, rc))
        c.reset()
        vis0, counts0 = c.visibilities()
        assert not vis0.any() and not counts0.any()


def test_invalid_calls_return_status():
    job = synth.random_job(nant=3, npol=1, nchan=256, numffts=10, seed=3)
    with corr_for(job) as c:
        with pytest.raises(fx.FxcError) as e:
            c.process(job.data, job.delays, job.fileoffsets, 5, 6)
        assert e.value.status == fx.FXC_ERR_INVALID
        bad = job.delays.copy()
        bad[1, 2] = np.nan
        with pytest.raises(fx.FxcError) as e:
            c.process(job.data, bad, job.fileoffsets)
        assert e.value.status == fx.FXC_ERR_INVALID
        c.process(job.data, job.delays, job.fileoffsets)   # context still usable
        c.synchronize()


# ---------------------------------------------------------------- tensor-core form
TC_RMS_TOL = 1e-3    # FP16 inputs, FP32 accumulation: RMS relative error per spectrum vs FP64
TC_MAX_TOL = 1e-2    # max |d| / max |ref| per spectrum


@pytest.mark.parametrize("nant,npol,nchan,nsb,numffts", [(4, 1, 256, 1, 64), (16, 2, 512, 2, 64),
                                                          (64, 1, 1024, 1, 64), (12, 1, 2048, 1, 32),
                                                          (33, 1, 128, 2, 128)])
def test_tc_vis_vs_fp64_oracle(nant, npol, nchan, nsb, numffts):
    job = synth.make_job(nant=nant, npol=npol, nchan=nchan, numffts=numffts, bw=64e6, lo=1.4e9, rho=0.1,
                         seed=nant * 7 + nchan, nsubband=nsb)
    with corr_for(job, xmode=fx.FXC_X_TC_FP16) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    for sb in range(nsb):
        ref, rc = oracle_vis(job, sb)
        np.testing.assert_array_equal(counts, rc)
        mx, rms = fo.vis_error(vis[sb], ref)
        assert rms.max() < TC_RMS_TOL, f"rms {rms.max():.3e}"
        assert mx.max() < TC_MAX_TOL, f"max {mx.max():.3e}"


@pytest.mark.parametrize("nant,npol,nchan,nsb,numffts,chunk,calls",
                         [(8, 2, 256, 2, 300, 128, [(0, 150), (150, 150)]),
                          (64, 1, 1024, 1, 256, 0, [(0, 256)]),
                          (5, 2, 4096, 1, 100, 0, [(0, 100)]),
                          (3, 1, 128, 3, 200, 64, [(0, 77), (77, 123)]),
                          (33, 1, 512, 1, 130, 0, [(0, 130)])])
def test_tc_fp32_spectra_path_bit_identical(nant, npol, nchan, nsb, numffts, chunk, calls, monkeypatch):
    """The FP16 tensor-core form of up to 64 signals reads the FFT F stage's FP32 spectra and casts
    to FP16 in the X stage; with FXC_TC_SPECTRA=f16 the F stage writes the FP16 K-major layout
    instead.  Same FP16 values, same MMAs in the same order: the same visibilities, bit for bit."""
    job = synth.make_job(nant=nant, npol=npol, nchan=nchan, numffts=numffts, bw=64e6, lo=1.4e9, rho=0.1,
                         seed=nant * 11 + nchan, nsubband=nsb)
    out = {}
    for layout in ("f32", "f16"):
        if layout == "f16":
            monkeypatch.setenv("FXC_TC_SPECTRA", "f16")
        else:
            monkeypatch.delenv("FXC_TC_SPECTRA", raising=False)
        with corr_for(job, xmode=fx.FXC_X_TC_FP16, chunk_ffts=chunk) as c:
            for first, n in calls:
                c.process(job.data, job.delays, job.fileoffsets, first, n)
            out[layout] = c.visibilities()
    np.testing.assert_array_equal(out["f32"][1], out["f16"][1])
    np.testing.assert_array_equal(out["f32"][0], out["f16"][0])
    ref, _ = oracle_vis(job, 0)
    mx, rms = fo.vis_error(out["f32"][0][0], ref)
    assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL


def test_tc_matches_plain_and_accumulates_over_chunks():
    job = synth.make_job(nant=24, npol=1, nchan=1024, numffts=300, bw=64e6, lo=1.4e9, rho=0.1, seed=31)
    out = {}
    for mode in (fx.FXC_X_PLAIN_FP32, fx.FXC_X_TC_FP16):
        with corr_for(job, xmode=mode, chunk_ffts=128) as c:
            c.process(job.data, job.delays, job.fileoffsets, 0, 150)
            c.process(job.data, job.delays, job.fileoffsets, 150, 150)
            out[mode] = c.visibilities(normalize=True)
    np.testing.assert_array_equal(out[0][1], out[1][1])
    mx, rms = fo.vis_error(out[1][0][0], out[0][0][0])
    assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL


# ---------------------------------------------------------------- FP8-E4M3 tensor-core form
E4M3_U = 2.0 ** -4 + 2.0 ** -11   # e4m3 unit roundoff, compounded with the F16 rounding before the cast
E4M3_SUB = 2.0 ** -10             # absolute rounding of e4m3 subnormals, in scaled units


def fp8_error_bound(job, sb, T):
    """Worst-case |V_fp8 - V| per product and channel from the quantisation model.

    Every spectrum value x of signal s, channel c in chunk k is stored as
    q = e4m3(x * 448 / amax[k][s][c]) with amax = max(|Re|, |Im|) over the chunk,
    so each component carries |err| <= u |x| + 2^-10 amax / 448 and the product
    x_i conj(x_j) carries |err| <= e_i |x_j| + |x_i| e_j + e_i e_j with
    e = u |x| + sqrt(2) 2^-10 amax / 448.  Returned in the visibility layout
    [nbl + nant][npol^2][nchan].
    """
    spec, _ = fo.channelise(job.data[sb], job.delays, job.fileoffsets, job.bw, float(job.sb_lo[sb]), job.nchan,
                            job.npol, np.arange(job.numffts), job.numffts)
    nsig = job.nant * job.npol
    X = spec.reshape(nsig, job.numffts, job.nchan)
    ax = np.abs(X)
    B = np.zeros((job.nchan, nsig, nsig))
    for t0 in range(0, job.numffts, T):
        xs = X[:, t0:t0 + T]
        a = ax[:, t0:t0 + T]
        amax = np.maximum(np.abs(xs.real), np.abs(xs.imag)).max(axis=1)        # [sig][chan]
        e = E4M3_U * a + np.sqrt(2.0) * E4M3_SUB * (amax / 448.0)[:, None, :]
        At, Et = a.transpose(2, 0, 1), e.transpose(2, 0, 1)                    # [chan][sig][t]
        B += Et @ At.transpose(0, 2, 1) + At @ Et.transpose(0, 2, 1) + Et @ Et.transpose(0, 2, 1)
    bls = fo.baseline_order(job.nant) + [(k, k) for k in range(job.nant)]
    out = np.zeros((len(bls), job.npol ** 2, job.nchan))
    for bi, (j, k) in enumerate(bls):
        for l in range(job.npol):
            for m in range(job.npol):
                out[bi, l * job.npol + m] = B[:, j * job.npol + l, k * job.npol + m]
    return out


@pytest.mark.parametrize("nant,npol,nchan,nsb,numffts,chunk", [(4, 1, 256, 1, 128, 0), (16, 2, 512, 2, 300, 128),
                                                                (64, 1, 1024, 1, 128, 0), (33, 1, 128, 2, 200, 128),
                                                                (8, 2, 1024, 1, 256, 256)])
def test_fp8_vis_within_quantisation_bound(nant, npol, nchan, nsb, numffts, chunk):
    job = synth.make_job(nant=nant, npol=npol, nchan=nchan, numffts=numffts, bw=64e6, lo=1.4e9, rho=0.1,
                         seed=nant * 11 + nchan, nsubband=nsb)
    with corr_for(job, xmode=fx.FXC_X_TC_FP8, chunk_ffts=chunk) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    T = chunk if chunk else int(np.ceil(numffts / 128) * 128)
    for sb in range(nsb):
        ref, rc = oracle_vis(job, sb)
        np.testing.assert_array_equal(counts, rc)
        bound = fp8_error_bound(job, sb, T)
        err = np.abs(vis[sb] - ref)
        # the bound is a worst case; FP32 F-stage and accumulation rounding add ~1e-6 relative
        slack = 1e-5 * np.abs(ref).max(axis=-1, keepdims=True)
        assert (err <= 1.01 * bound + slack).all(), f"sb {sb}: max err/bound {(err / (bound + slack)).max():.3f}"
        mx, rms = fo.vis_error(vis[sb], ref)
        assert rms.max() < 0.05       # loose sanity bound; the per-product bound above is the contract


def test_fp8_accumulates_over_calls_like_plain():
    job = synth.make_job(nant=24, npol=1, nchan=1024, numffts=512, bw=64e6, lo=1.4e9, rho=0.1, seed=37)
    out = {}
    for mode in (fx.FXC_X_PLAIN_FP32, fx.FXC_X_TC_FP8):
        with corr_for(job, xmode=mode, chunk_ffts=256) as c:
            c.process(job.data, job.delays, job.fileoffsets, 0, 256)
            c.process(job.data, job.delays, job.fileoffsets, 256, 256)
            out[mode] = c.visibilities(normalize=True)
    np.testing.assert_array_equal(out[0][1], out[2][1])
    mx, rms = fo.vis_error(out[2][0][0], out[0][0][0])
    assert rms.max() < 0.05


@pytest.mark.parametrize("xmode", [fx.FXC_X_PLAIN_FP32, fx.FXC_X_TC_FP16])
def test_plans_change_speed_not_results(xmode, tmp_path, monkeypatch):
    job = synth.make_job(nant=12, npol=2, nchan=512, numffts=256, bw=64e6, lo=1.4e9, rho=0.1, seed=77)
    ref = None
    with corr_for(job, xmode=xmode) as c:
        for tb, alt in [(16, 0), (8, 1), (32, 0)]:
            c.set_plan(tb, alt)
            c.reset()
            c.process(job.data, job.delays, job.fileoffsets)
            vis = c.visibilities()[0]
            if ref is None:
                ref = vis
            else:
                np.testing.assert_array_equal(vis, ref)
        with pytest.raises(fx.FxcError):
            c.set_plan(12, 0)
        cache = tmp_path / "plans.txt"
        monkeypatch.setenv("FXC_PLAN_CACHE", str(cache))
        c.autotune(reps=2)
        tuned = c.plan()
        c.process(job.data, job.delays, job.fileoffsets)
        np.testing.assert_array_equal(c.visibilities()[0], ref)
    key = ("F " if xmode == fx.FXC_X_PLAIN_FP32 else "H ") + "1024 2 "
    assert any(line.startswith(key) for line in cache.read_text().splitlines())
    with corr_for(job, xmode=xmode) as c2:
        assert c2.plan() == tuned


# ---------------------------------------------------------------- multi-block Gram (65..512 signals)
@pytest.mark.parametrize("nant,npol,nchan,numffts,xmode", [
    (48, 2, 512, 64, fx.FXC_X_TC_FP16),     # 96 signals: 1 x 128-row block + padding
    (65, 2, 256, 64, fx.FXC_X_TC_FP16),     # 130 signals: 3 blocks, odd padding
    (200, 1, 128, 128, fx.FXC_X_TC_FP16),   # 4 blocks
    (256, 2, 128, 64, fx.FXC_X_TC_FP16),    # 512 signals: 8 blocks, 36 block pairs per channel
    (80, 2, 256, 128, fx.FXC_X_TC_FP8),
])
def test_tc_multiblock_vs_fp64_oracle(nant, npol, nchan, numffts, xmode):
    job = synth.make_job(nant=nant, npol=npol, nchan=nchan, numffts=numffts, bw=64e6, lo=1.4e9, rho=0.1,
                         seed=nant + nchan)
    with corr_for(job, xmode=xmode) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    ref, rc = oracle_vis(job)
    np.testing.assert_array_equal(counts, rc)
    if xmode == fx.FXC_X_TC_FP16:
        mx, rms = fo.vis_error(vis[0], ref)
        assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL, f"rms {rms.max():.3e} max {mx.max():.3e}"
    else:
        bound = fp8_error_bound(job, 0, int(np.ceil(numffts / 128) * 128))
        err = np.abs(vis[0] - ref)
        slack = 1e-5 * np.abs(ref).max(axis=-1, keepdims=True)
        assert (err <= 1.01 * bound + slack).all()


@pytest.mark.parametrize("nant,npol,nchan,numffts,nsb", [(48, 2, 256, 64, 1), (65, 2, 128, 64, 2),
                                                          (200, 1, 128, 64, 1)])
def test_plain_multiblock_vs_fp64_oracle(nant, npol, nchan, numffts, nsb):
    job = synth.make_job(nant=nant, npol=npol, nchan=nchan, numffts=numffts, bw=64e6, lo=1.4e9, rho=0.1,
                         seed=3 * nant + nchan, nsubband=nsb)
    with corr_for(job) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    for sb in range(nsb):
        ref, rc = oracle_vis(job, sb)
        np.testing.assert_array_equal(counts, rc)
        assert_vis_close(vis[sb], ref)


@pytest.mark.parametrize("nant,npol,nchan,numffts,nsb,chunk,calls",
                         [(4, 1, 256, 1000, 1, 0, [(0, 1000)]),
                          (6, 2, 128, 700, 2, 512, [(0, 300), (300, 400)]),
                          (8, 1, 512, 640, 1, 256, [(0, 129), (129, 511)])])
def test_plain_time_segments_vs_fp64_oracle(nant, npol, nchan, numffts, nsb, chunk, calls):
    """Few channel groups: the plain X stage cuts the FFT slots into time segments, sums each
    segment into its own partials and reduces them into the accumulator (chunks that fill only
    some segments, calls that split a chunk)."""
    job = synth.make_job(nant=nant, npol=npol, nchan=nchan, numffts=numffts, bw=64e6, lo=1.4e9, rho=0.1,
                         seed=nant + nchan + numffts, nsubband=nsb)
    with corr_for(job, chunk_ffts=chunk) as c:
        for first, n in calls:
            c.process(job.data, job.delays, job.fileoffsets, first, n)
        vis, counts = c.visibilities()
    for sb in range(nsb):
        ref, rc = oracle_vis(job, sb)
        np.testing.assert_array_equal(counts, rc)
        assert_vis_close(vis[sb], ref)


def test_tc_matches_plain_multiblock():
    job = synth.make_job(nant=70, npol=2, nchan=256, numffts=256, bw=64e6, lo=1.4e9, rho=0.1, seed=71)
    out = {}
    for mode in (fx.FXC_X_PLAIN_FP32, fx.FXC_X_TC_FP16):
        with corr_for(job, xmode=mode, chunk_ffts=128) as c:
            c.process(job.data, job.delays, job.fileoffsets)
            out[mode] = c.visibilities(normalize=True)
    np.testing.assert_array_equal(out[0][1], out[1][1])
    mx, rms = fo.vis_error(out[1][0][0], out[0][0][0])
    assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL


@pytest.mark.parametrize("nant,npol,nchan,xmode", [(4, 2, 4096, fx.FXC_X_TC_FP16), (5, 2, 2048, fx.FXC_X_TC_FP16),
                                                   (4, 1, 4096, fx.FXC_X_TC_FP16), (3, 2, 4096, fx.FXC_X_TC_FP8)])
def test_tc_long_ffts_dual_pol(nant, npol, nchan, xmode):
    """FFT length x polarisations beyond what 16 FFTs of F16 staging hold: fewer FFTs per CTA."""
    job = synth.make_job(nant=nant, npol=npol, nchan=nchan, numffts=128, bw=64e6, lo=1.4e9, rho=0.1,
                         seed=nchan + npol)
    with corr_for(job, xmode=xmode) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    ref, rc = oracle_vis(job)
    np.testing.assert_array_equal(counts, rc)
    if xmode == fx.FXC_X_TC_FP16:
        mx, rms = fo.vis_error(vis[0], ref)
        assert rms.max() < TC_RMS_TOL and mx.max() < TC_MAX_TOL
    else:
        bound = fp8_error_bound(job, 0, 128)
        slack = 1e-5 * np.abs(ref).max(axis=-1, keepdims=True)
        assert (np.abs(vis[0] - ref) <= 1.01 * bound + slack).all()


def test_expired_device_wait_is_reported_and_context_survives():
    """A bounded device wait that runs out (on a barrier nothing completes) comes back as
    FXC_ERR_TIMEOUT with its code; the next correlation on the same context is correct."""
    import ctypes as C
    job = synth.make_job(nant=4, npol=1, nchan=256, numffts=64, bw=64e6, lo=1.4e9, rho=0.1, seed=91)
    with corr_for(job) as c:
        assert fx.lib().fxc_debug_expire_wait(C.c_void_p(c.handle.value)) == fx.FXC_OK
        with pytest.raises(fx.FxcError) as e:
            c.synchronize()
        assert e.value.status == fx.FXC_ERR_TIMEOUT
        assert fx.lib().fxc_last_device_error() == 6
        c.reset()
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    ref, rc = oracle_vis(job)
    np.testing.assert_array_equal(counts, rc)
    assert_vis_close(vis[0], ref)
