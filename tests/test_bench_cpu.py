"""CPU checks of bench.py's reference sampling: the reference CPU correlator reads only
interleaved dual-polarisation input with a square channel count, so each workload's CPU
baseline and reference arm run the reference on a dual-pol geometry it accepts, stated in
the sample description."""
import math
import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402


def test_reference_geometry_per_workload():
    g0 = bench.ref_geom_for("cfg0")
    assert (g0["nant"], g0["nchan"]) == (4, 256)          # the dual-pol variant of cfg0
    assert "4 ant x 2 pol" in bench.ref_workload_desc(10)
    for wl in ("cfg1", "cfg2", "cfg4", "cfg3"):
        g = bench.ref_geom_for(wl)
        assert (g["nant"], g["nchan"]) == (32, 1024)      # 64 signals as 32 dual-pol antennas
    for g in bench.REF_GEOMS.values():
        assert math.isqrt(g["nchan"]) ** 2 == g["nchan"]  # kernel.c:31-35 needs a square channel count
    bench.ref_geom_for("cfg2")


def test_forms_headline_first_and_geometry_fallback():
    w2 = bench.WORKLOADS["cfg2"]
    assert bench.select_forms("all", w2) == ["tc32f", "tc", "tc16f", "fp8", "plain"]
    assert bench.select_forms("both", w2) == ["tc32f", "plain"]
    # 2048 channels x 2 pol: no tensor-core F stage, the FP32 FFT form leads
    w1 = bench.WORKLOADS["cfg1"]
    assert bench.select_forms("all", w1) == ["tc", "fp8", "plain"]
    assert bench.select_forms("both", w1) == ["tc", "plain"]
    assert bench.select_forms("plain", w1) == ["plain"]
    for f, (xmode, fstage) in bench.FORMS.items():
        assert f in bench.DTYPES and fstage in bench.F_KERNELS


def test_form_parameters_fall_back_where_the_tensor_core_f_stages_do_not_apply():
    w2, w1 = bench.WORKLOADS["cfg2"], bench.WORKLOADS["cfg1"]
    assert bench.form_params("tc32f", w2) == (1, 3) and bench.form_params("tc16f", w2) == (1, 2)
    assert bench.form_params("tc32f", w1) == (1, 1) and bench.form_params("fp8", w1) == (2, 1)
    assert "k_ftc32" in bench.form_dtype("tc32f", w2) and "FFT" in bench.form_dtype("tc32f", w1)


def test_spectra_layout_follows_the_library_rule(monkeypatch):
    """The F stage writes FP32 spectra for the FP16 tensor-core form on the FFT at up to 64 signals
    (its X stage casts them), FP16 K-major for the other tensor-core forms and geometries."""
    monkeypatch.delenv("FXC_TC_SPECTRA", raising=False)
    w1, w2 = bench.WORKLOADS["cfg1"], bench.WORKLOADS["cfg2"]
    w4 = dict(w1, nant=256)                                 # the large array: 512 signals
    assert not bench.spectra_f16(0, 1, w2)                 # plain
    assert not bench.spectra_f16(1, 1, w1) and not bench.spectra_f16(1, 1, w2)   # tc on the FFT
    assert bench.spectra_f16(1, 3, w2) and bench.spectra_f16(1, 2, w2)          # tensor-core F stages
    assert bench.spectra_f16(2, 1, w2)                      # FP8
    assert bench.spectra_f16(1, 1, w4)                      # 512 signals
    monkeypatch.setenv("FXC_TC_SPECTRA", "f16")
    assert bench.spectra_f16(1, 1, w1)
