"""CPU tests of the C ABI: the library loads, exports every declared symbol and
validates arguments on the host (no GPU compute is called here)."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

import difx_tests_b200 as fx

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", src, flags=re.M):
            name = m.group(1)
            if name not in ("if", "defined"):
                names.add(name)
    return names


def exported_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_exports_every_declared_symbol():
    decl = declared_functions()
    assert "fxc_create" in decl and "fxc_process_host" in decl
    exported = exported_symbols(fx.LIB_PATH)
    missing = sorted(decl - exported)
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_abi():
    fx.lib()
    decl = {n for n in declared_functions() if n.startswith("fxc_")}
    assert decl <= set(fx.SIGNATURES), sorted(decl - set(fx.SIGNATURES))


def test_config_helpers():
    L = fx.lib()
    cfg = fx.make_config(4, 256, 3125, 32e6, 1.4e9, npol=1)
    # allocDataHost.c:21: nchan * 2 * (numffts + 1) * nbit / 8 * npol
    assert L.fxc_subint_bytes(C.byref(cfg)) == 256 * 2 * 3126 * 2 // 8
    assert L.fxc_num_baselines(C.byref(cfg)) == 6
    assert L.fxc_vis_count(C.byref(cfg)) == (6 + 4) * 1 * 256
    cfg2 = fx.make_config(16, 2048, 31250, 64e6, 1.4e9, npol=2, nsubband=4)
    assert L.fxc_vis_count(C.byref(cfg2)) == 4 * (120 + 16) * 4 * 2048


@pytest.mark.parametrize("field,value,status", [
    ("nant", 1, fx.FXC_ERR_INVALID),
    ("nant", 257, fx.FXC_ERR_UNSUPPORTED),    # 514 signals at npol 2
    ("nchan", 300, fx.FXC_ERR_INVALID),
    ("nchan", 64, fx.FXC_ERR_INVALID),
    ("npol", 3, fx.FXC_ERR_INVALID),
    ("nbit", 8, fx.FXC_ERR_UNSUPPORTED),
    ("iscomplex", 1, fx.FXC_ERR_UNSUPPORTED),
    ("chunk_ffts", 100, fx.FXC_ERR_INVALID),
    ("bw", 0.0, fx.FXC_ERR_INVALID),
])
def test_invalid_config_rejected_before_device_use(field, value, status):
    cfg = fx.make_config(4, 256, 64, 32e6, 1.4e9)
    setattr(cfg, field, value)
    ctx = C.c_void_p()
    assert fx.lib().fxc_create(C.byref(cfg), C.byref(ctx)) == status
    assert not ctx.value


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_create_without_device_returns_status():
    cfg = fx.make_config(4, 256, 64, 32e6, 1.4e9)
    with pytest.raises(fx.FxcError) as e:
        fx.Correlator(cfg)
    assert e.value.status in (fx.FXC_ERR_CUDA, fx.FXC_ERR_NODEVICE)


def test_null_arguments_rejected():
    L = fx.lib()
    assert L.fxc_create(None, None) == fx.FXC_ERR_INVALID
    assert L.fxc_reset(None) == fx.FXC_ERR_INVALID
    assert L.fxc_process_host(None, None, None, None, 0, 1) == fx.FXC_ERR_INVALID
    assert L.fxc_get_visibilities(None, None, None, 0) == fx.FXC_ERR_INVALID
    assert L.fxc_get_amp_phase(None, None, 0) == fx.FXC_ERR_INVALID
    assert L.fxc_strerror(fx.FXC_ERR_NOMEM).decode().startswith("out of")


def test_batch_arguments_rejected():
    L = fx.lib()
    out = C.c_void_p()
    cfg = fx.make_config(4, 256, 64, 32e6, 1.4e9)
    assert L.fxc_batch_create(None, 1, C.byref(out)) == fx.FXC_ERR_INVALID
    assert L.fxc_batch_create(C.byref(cfg), 0, C.byref(out)) == fx.FXC_ERR_INVALID
    # forms the batch does not run: FP8 X, input windows, the tensor-core F stages
    for kw in (dict(xmode=fx.FXC_X_TC_FP8), dict(window_ffts=64), dict(fstage=fx.FXC_F_TC32)):
        unsup = fx.make_config(4, 256, 64, 32e6, 1.4e9, **kw)
        assert L.fxc_batch_create(C.byref(unsup), 1, C.byref(out)) == fx.FXC_ERR_UNSUPPORTED
    bad = fx.make_config(4, 300, 64, 32e6, 1.4e9)
    assert L.fxc_batch_create(C.byref(bad), 1, C.byref(out)) == fx.FXC_ERR_INVALID
    assert not out.value
    assert L.fxc_batch_process(None) == fx.FXC_ERR_INVALID
    assert L.fxc_batch_reset(None) == fx.FXC_ERR_INVALID
    assert L.fxc_batch_autotune(None, 1) == fx.FXC_ERR_INVALID
    assert L.fxc_batch_get_visibilities(None, 0, None, None, 0) == fx.FXC_ERR_INVALID
    assert L.fxc_batch_upload(None, 0, None) == fx.FXC_ERR_INVALID
    assert L.fxc_batch_set_model(None, 0, None, None) == fx.FXC_ERR_INVALID
    L.fxc_batch_destroy(None)


def test_fp8_form_config_rules():
    L = fx.lib()
    ctx = C.c_void_p()
    cfg = fx.make_config(4, 256, 64, 32e6, 1.4e9, xmode=fx.FXC_X_TC_FP8, chunk_ffts=64)
    assert L.fxc_create(C.byref(cfg), C.byref(ctx)) == fx.FXC_ERR_INVALID      # FP8 chunks are 128-FFT multiples
    cfg = fx.make_config(4, 256, 64, 32e6, 1.4e9, xmode=3)
    assert L.fxc_create(C.byref(cfg), C.byref(ctx)) == fx.FXC_ERR_INVALID
    assert not ctx.value


def test_plan_arguments_rejected():
    L = fx.lib()
    assert L.fxc_set_plan(None, 16, 0) == fx.FXC_ERR_INVALID
    assert L.fxc_get_plan(None, None, None) == fx.FXC_ERR_INVALID
    assert L.fxc_autotune(None, 1) == fx.FXC_ERR_INVALID


def test_complex_input_config_rules():
    L = fx.lib()
    ctx = C.c_void_p()
    cfg = fx.make_config(4, 128, 64, 32e6, 1.4e9, cpx=True)
    assert L.fxc_create(C.byref(cfg), C.byref(ctx)) == fx.FXC_ERR_UNSUPPORTED     # complex FFT length >= 256
    cfg = fx.make_config(4, 256, 64, 32e6, 1.4e9)
    cfg.nbit = 8                                                                   # 8-bit real: not a format
    assert L.fxc_create(C.byref(cfg), C.byref(ctx)) == fx.FXC_ERR_UNSUPPORTED
    cfg = fx.make_config(4, 1024, 99, 32e6, 1.4e9, npol=2, cpx=True)
    assert L.fxc_subint_bytes(C.byref(cfg)) == 1024 * 100 * 4
    assert not ctx.value
