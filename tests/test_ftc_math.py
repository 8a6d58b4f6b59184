"""CPU check of the tensor-core F stage's arithmetic (difx_tests_b200/csrc/fx_ftc.cu), restated
with numpy: the 2048-point DFT as step 1 (a 32-point DFT over n1 as a real-form GEMM), twiddles
W2048^(n2 k1), step 2 (a 64-point DFT over n2 as a real-form GEMM, channels k2 < 32 only) and the
fractional-sample factor fsub[k1] * fstep[k2].  In FP64 it reproduces the FFT's first 1024
channels to rounding; with FP16 operands and intermediates at the points where the kernel rounds
(rotated samples, DFT matrices, twiddled intermediate, output) the spectra stay within a few
1e-4 relative RMS, the error budget behind the tensor-core form's bar (RMS <= 1e-3 on the
visibilities)."""
import numpy as np

F, F1, F2, C = 2048, 32, 64, 1024


def real_form(w):
    """Real form of a complex matrix W[n_out][k_in]: rows (out, re|im), columns (in, re|im), so
    that y = W x becomes [yr, yi] interleaved = R . [xr, xi] interleaved (the B-operand layout)."""
    n, k = w.shape
    r = np.zeros((2 * n, 2 * k))
    r[0::2, 0::2] = w.real
    r[0::2, 1::2] = -w.imag
    r[1::2, 0::2] = w.imag
    r[1::2, 1::2] = w.real
    return r


def interleave(z):
    out = np.empty(z.shape[:-1] + (2 * z.shape[-1],))
    out[..., 0::2] = z.real
    out[..., 1::2] = z.imag
    return out


def deinterleave(a):
    return a[..., 0::2] + 1j * a[..., 1::2]


def ftc_spectrum(x, fs, fst, half=None):
    """One FFT's 1024 channels the way k_ftc computes them; `half` = rounding function (None: exact)."""
    q = half or (lambda v: v)
    n1, n2, k1, k2 = np.arange(F1), np.arange(F2), np.arange(F1), np.arange(C // F1)
    b1 = q(real_form(np.exp(-2j * np.pi * np.outer(k1, n1) / F1)))            # [(k1,c)][(n1,c')]
    b2 = q(real_form(np.exp(-2j * np.pi * np.outer(k2, n2) / F2)))            # [(k2,c)][(n2,c')]
    tw = np.exp(-2j * np.pi * np.outer(n2, k1) / F)                           # [n2][k1]
    a1 = q(interleave(x.reshape(F1, F2).T))                                    # rows n2, K = (n1, re|im)
    y = deinterleave(a1 @ b1.T)                                                # D1[n2][k1]
    z = q(interleave((y * tw).T))                                              # A2 rows k1, K = (n2, re|im)
    xk = deinterleave(z @ b2.T)                                                # D2[k1][k2]
    out = xk * np.outer(fs, fst)                                               # fsub[k1] fstep[k2]
    return q(interleave(out.T.reshape(-1)))                                    # channel k = k1 + 32 k2


def test_factorisation_is_the_dft_and_fp16_error_budget():
    rng = np.random.default_rng(7)
    levels = np.array([-3.3359, -1.0, 1.0, 3.3359])
    lv = levels[rng.integers(0, 4, F)]
    # fringe rotator sub[n % 64] * step[n / 64] and fractional-sample factors with random phases
    sub = np.exp(1j * rng.uniform(-np.pi, np.pi, F2))
    step = np.exp(1j * rng.uniform(-np.pi, np.pi, F1))
    x = lv * (sub[np.arange(F) % F2] * step[np.arange(F) // F2])
    fs = np.exp(1j * rng.uniform(-np.pi, np.pi, F1))
    fst = np.exp(1j * rng.uniform(-np.pi, np.pi, C // F1))
    k = np.arange(C)
    ref = np.fft.fft(x)[:C] * fs[k % F1] * fst[k // F1]

    exact = deinterleave(ftc_spectrum(x, fs, fst))
    assert np.abs(exact - ref).max() <= 1e-9 * np.abs(ref).max()

    def half(v):
        return np.asarray(v, np.float16).astype(np.float64)

    got = deinterleave(ftc_spectrum(x, fs, fst, half))
    rms = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert rms < 1e-3, rms
    assert rms > 1e-5                 # the FP16 roundings are really applied


# ---------------------------------------------------------------------------------------------
# FP32-grade tensor-core F stage (error-compensated FP16 split).  Every FP16 operand is a pair
# hi + lo (hi = FP16 rounding, or for the twiddled intermediate the value truncated to 11
# significant bits, lo = FP16 rounding of the remainder) and each GEMM is the three
# products hi.hi + lo.hi + hi.lo accumulated in FP32 (the lo.lo term is below FP32 rounding).
# The fringe rotator is split as the reference builds it (kernel.c:428-497): the step factor of
# n1 goes into the step-1 operand through a per-(FFT, n1) table of the four levels times step[n1]
# (so the operand is an exact hi/lo pair of the FP32 product), the sub factor of n2 and the
# fractional-sample factor fsub[k1] (kernel.c:512-555) ride on the twiddle W2048^(n2 k1), evaluated
# per row n2 by a complex recurrence over k1 restarted at k1 = 16, and fstep[k2] is applied to the
# step-2 output.  FP32 arithmetic everywhere else.

def split16(v):
    """(hi, lo) FP16 pair of a float32 array: hi = RN16(v), lo = RN16(v - hi)."""
    v = np.asarray(v, np.float32)
    hi = v.astype(np.float16)
    lo = (v - hi.astype(np.float32)).astype(np.float16)
    return hi.astype(np.float64), lo.astype(np.float64)


def split16t(v):
    """The twiddle stage's pair: hi = v truncated to 11 significant bits (exact in FP16),
    lo = RN16(v - hi)."""
    v = np.asarray(v, np.float32)
    hi = (v.view(np.uint32) & np.uint32(0xFFFFE000)).view(np.float32)
    return hi.astype(np.float16).astype(np.float64), (v - hi).astype(np.float16).astype(np.float64)


def gemm3(a, b):
    """A . B^T with A, B split into FP16 pairs: hi.hi + lo.hi + hi.lo (FP32-accumulated products
    are exact in FP64 here; the accumulation order does not matter at this precision)."""
    ah, al = a
    bh, bl = b
    return ah @ bh.T + al @ bh.T + ah @ bl.T


def cmul32(a, b):
    return (np.asarray(a, np.complex64) * np.asarray(b, np.complex64)).astype(np.complex64)


def ftc32_spectrum(codes, levels, sub, step, theta):
    """One FFT's 1024 channels the way the FP32-grade tensor-core F stage computes them.
    codes [F] 2-bit codes, sub [64] / step [32] fringe factors, theta: fractional-sample phase
    step per channel (fsub[k1] = e^{i theta k1}, fstep[k2] = e^{i theta 32 k2})."""
    n1, n2, k1, k2 = np.arange(F1), np.arange(F2), np.arange(F1), np.arange(C // F1)
    # step-1 operand: table[n1][code] = level(code) * step[n1] in FP32, split
    table = cmul32(levels[None, :].astype(np.complex64), step[:, None])            # [n1][code]
    x = table[n1[None, :], codes.reshape(F1, F2).T]                                  # [n2][n1]
    xr = interleave(x.astype(np.complex128)).astype(np.float32)                      # rows n2, K (n1, c)
    b1 = real_form(np.exp(-2j * np.pi * np.outer(k1, n1) / F1)).astype(np.float32)  # [(k1,c)][(n1,c')]
    y = deinterleave(gemm3(split16(xr), split16(b1))).astype(np.complex64)          # D1[n2][k1], FP32
    # twiddle sub[n2] * W2048^(n2 k1) * fsub[k1] by recurrence over k1, restarted at k1 = 16
    rho = np.exp(1j * (-2 * np.pi * n2 / F + theta)).astype(np.complex64)           # per row
    t = np.empty((F2, F1), np.complex64)
    for start in (0, 16):
        cur = cmul32(sub, np.exp(1j * (-2 * np.pi * n2 * start / F + theta * start)))
        for j in range(16):
            t[:, start + j] = cur
            cur = cmul32(cur, rho)
    z = cmul32(y, t)                                                                 # [n2][k1]
    zr = interleave(z.T.astype(np.complex128)).astype(np.float32)                   # rows k1, K (n2, c)
    b2 = real_form(np.exp(-2j * np.pi * np.outer(k2, n2) / F2)).astype(np.float32)  # [(k2,c)][(n2,c')]
    xk = deinterleave(gemm3(split16t(zr), split16(b2))).astype(np.complex64)        # D2[k1][k2]
    fst = np.exp(1j * theta * F1 * k2).astype(np.complex64)
    out = cmul32(xk, fst[None, :])                                                   # fstep[k2]
    return out.T.reshape(-1)                                                         # channel k1 + 32 k2


def test_fp32_grade_split_meets_the_fp32_spectra_bar():
    """The FP32 F stage's bar (spectra within 2e-5 of max|X| per spectrum vs FP64, the bar the
    FP32 FFT kernel is held to) holds for the three-product FP16 split, on noise-like levels and
    on a strong tone (a large dynamic range inside one spectrum)."""
    rng = np.random.default_rng(11)
    levels = np.array([-3.3359, -1.0, 1.0, 3.3359], np.float32)
    worst = 0.0
    for trial in range(6):
        if trial < 4:
            codes = rng.integers(0, 4, F)
        else:   # a tone plus noise, quantised: a spectrum with one dominant channel
            n = np.arange(F)
            s = 3.0 * np.cos(2 * np.pi * 123.3 * n / F + 0.4) + rng.standard_normal(F)
            codes = np.digitize(s, [-0.98, 0.0, 0.98])
        sub = np.exp(1j * rng.uniform(-np.pi, np.pi, F2)).astype(np.complex64)
        step = np.exp(1j * rng.uniform(-np.pi, np.pi, F1)).astype(np.complex64)
        theta = rng.uniform(-np.pi, np.pi) / C
        x = levels[codes].astype(np.float64) * sub[np.arange(F) % F2] * step[np.arange(F) // F2]
        k = np.arange(C)
        ref = np.fft.fft(x)[:C] * np.exp(1j * theta * k)
        got = ftc32_spectrum(codes, levels, sub, step, theta)
        err = np.abs(got - ref).max() / np.abs(ref).max()
        worst = max(worst, err)
        assert err < 2e-5, (trial, err)
    # and far below what one FP16 rounding of the operands gives (~3e-4 RMS)
    assert worst < 2e-6, worst
