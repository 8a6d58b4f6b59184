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
