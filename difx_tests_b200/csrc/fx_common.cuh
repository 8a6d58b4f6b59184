// fx_common.cuh -- shared device helpers for the B200 FX correlator.
//
// Complex float2 arithmetic, register-resident DFT building blocks (radix 2, 4,
// 8, 16; forward, e^{-i}, natural-order outputs) and IEEE binary64 helpers that
// forbid FMA contraction, so the delay/offset arithmetic reproduces the
// reference's x86-64 double results bit for bit (kernel.c:373-386, 733-756).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include "fx_internal.h"

namespace fx {

// Sets a kernel's dynamic shared-memory limit once per device (the attribute is
// per function and device).  `mask` is the caller's per-kernel static word.
template <typename Kern>
inline cudaError_t set_smem_once(Kern kern, size_t bytes, unsigned* mask)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned bit = 1u << (dev & 31);
    if (*mask & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) *mask |= bit;
    return e;
}

// Largest dynamic shared memory a block of the current device may opt in to.
inline size_t smem_optin_limit()
{
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
    return (size_t)v;
}

// Shared memory of one SM of the current device (all resident CTAs together).
inline size_t smem_per_sm_limit()
{
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess) return 0;
    return (size_t)v;
}

// ---------------------------------------------------------------- FP64 (no FMA)
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
// C's (int)x for in-range x: truncation toward zero.
__device__ __forceinline__ int dtrunc_int(double x) { return __double2int_rz(x); }
// x - (int)x, as the reference writes it (kernel.c:434-435, 465, 469).
__device__ __forceinline__ double dfrac_c(double x) { return dsub(x, (double)dtrunc_int(x)); }

// ------------------------------------------------------------------- complex
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * (-i)
__device__ __forceinline__ float2 cmul_mi(float2 a) { return make_float2(a.y, -a.x); }

// -------------------------------------------------------------- DFT blocks
// All transforms are forward (kernel sign e^{-2 pi i nk/N}) and leave outputs
// in natural order in the same array.
__device__ __forceinline__ void dft2(float2& a, float2& b)
{
    float2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3)
{
    float2 t0 = cadd(a0, a2), t1 = csub(a0, a2);
    float2 t2 = cadd(a1, a3), t3 = cmul_mi(csub(a1, a3));
    a0 = cadd(t0, t2);
    a2 = csub(t0, t2);
    a1 = cadd(t1, t3);
    a3 = csub(t1, t3);
}

constexpr float kSqrtHalf = 0.70710678118654752440f;
constexpr float kCos1_16 = 0.92387953251128675613f;  // cos(pi/8)
constexpr float kSin1_16 = 0.38268343236508977173f;  // sin(pi/8)

template <int R>
__device__ __forceinline__ void dft(float2* v);

template <>
__device__ __forceinline__ void dft<2>(float2* v) { dft2(v[0], v[1]); }

template <>
__device__ __forceinline__ void dft<4>(float2* v) { dft4(v[0], v[1], v[2], v[3]); }

template <>
__device__ __forceinline__ void dft<8>(float2* v)
{
    // radix-2 DIT over two 4-point transforms
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4(e0, e1, e2, e3);
    dft4(o0, o1, o2, o3);
    o1 = make_float2((o1.x + o1.y) * kSqrtHalf, (o1.y - o1.x) * kSqrtHalf);   // * W8^1
    o2 = cmul_mi(o2);                                                          // * W8^2
    o3 = make_float2((o3.y - o3.x) * kSqrtHalf, -(o3.x + o3.y) * kSqrtHalf);  // * W8^3
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

// W16^m for m = n2*k1 (n2, k1 in 1..3): forward twiddle e^{-2 pi i m / 16}
__device__ __forceinline__ float2 w16(int m)
{
    switch (m) {
    case 1: return make_float2(kCos1_16, -kSin1_16);
    case 2: return make_float2(kSqrtHalf, -kSqrtHalf);
    case 3: return make_float2(kSin1_16, -kCos1_16);
    case 4: return make_float2(0.f, -1.f);
    case 6: return make_float2(-kSqrtHalf, -kSqrtHalf);
    case 9: return make_float2(-kCos1_16, kSin1_16);
    default: return make_float2(1.f, 0.f);
    }
}

template <>
__device__ __forceinline__ void dft<16>(float2* v)
{
    // n = 4*n1 + n2, k = k1 + 4*k2
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) dft4(v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]);
    // now v[n2 + 4*k1] = Y[n2][k1]; twiddle by W16^{n2*k1}
#pragma unroll
    for (int n2 = 1; n2 < 4; n2++) {
#pragma unroll
        for (int k1 = 1; k1 < 4; k1++) {
            const int m = n2 * k1;
            if (m == 4) v[n2 + 4 * k1] = cmul_mi(v[n2 + 4 * k1]);
            else v[n2 + 4 * k1] = cmul(v[n2 + 4 * k1], w16(m));
        }
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) dft4(v[4 * k1 + 0], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    // v[4*k1 + k2] = X[k1 + 4*k2] -> transpose to natural order
    float2 t[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++)
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) t[k1 + 4 * k2] = v[4 * k1 + k2];
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = t[i];
}

// Forward DFT of R points keeping only outputs [0, R/2) (in v[0 .. R/2)): the
// last FFT pass needs channels below nchan = F/2 only.
template <int R>
__device__ __forceinline__ void dft_lo(float2* v);

template <>
__device__ __forceinline__ void dft_lo<2>(float2* v) { v[0] = cadd(v[0], v[1]); }

template <>
__device__ __forceinline__ void dft_lo<4>(float2* v)
{
    const float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const float2 t2 = cadd(v[1], v[3]), t3 = cmul_mi(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[1] = cadd(t1, t3);
}

template <>
__device__ __forceinline__ void dft_lo<8>(float2* v)
{
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4(e0, e1, e2, e3);
    dft4(o0, o1, o2, o3);
    o1 = make_float2((o1.x + o1.y) * kSqrtHalf, (o1.y - o1.x) * kSqrtHalf);
    o2 = cmul_mi(o2);
    o3 = make_float2((o3.y - o3.x) * kSqrtHalf, -(o3.x + o3.y) * kSqrtHalf);
    v[0] = cadd(e0, o0);
    v[1] = cadd(e1, o1);
    v[2] = cadd(e2, o2);
    v[3] = cadd(e3, o3);
}

template <>
__device__ __forceinline__ void dft_lo<16>(float2* v)
{
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) dft4(v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]);
#pragma unroll
    for (int n2 = 1; n2 < 4; n2++) {
#pragma unroll
        for (int k1 = 1; k1 < 4; k1++) {
            const int m = n2 * k1;
            if (m == 4) v[n2 + 4 * k1] = cmul_mi(v[n2 + 4 * k1]);
            else v[n2 + 4 * k1] = cmul(v[n2 + 4 * k1], w16(m));
        }
    }
    // X[k1 + 4*k2] for k2 in {0, 1}: outputs 0 and 1 of the 4-point DFT over n2
    float2 lo[4], hi[4];
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) {
        const float2 a0 = v[4 * k1 + 0], a1 = v[4 * k1 + 1], a2 = v[4 * k1 + 2], a3 = v[4 * k1 + 3];
        const float2 t0 = cadd(a0, a2), t1 = csub(a0, a2);
        const float2 t2 = cadd(a1, a3), t3 = cmul_mi(csub(a1, a3));
        lo[k1] = cadd(t0, t2);
        hi[k1] = cadd(t1, t3);
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) {
        v[k1] = lo[k1];
        v[k1 + 4] = hi[k1];
    }
}

// 2-bit code -> quantiser level {-HiMag, -1, +1, +HiMag} (kernel.c:191-200)
__device__ __forceinline__ float level2bit(uint32_t c)
{
    const float m = ((c + 1u) & 2u) ? 1.0f : kHiMag;
    return (c & 2u) ? m : -m;
}

}  // namespace fx
