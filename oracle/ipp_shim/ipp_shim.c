/*
 * ipp_shim.c -- from-scratch bodies for the Intel IPP entry points that the
 * reference CPU correlator uses.  TEST INFRASTRUCTURE ONLY: this builds the
 * oracle (the reference kernel.c/main.c compiled here, see oracle/Makefile);
 * nothing in the product links it.
 *
 * Semantics follow IPP's published documentation:
 *   - element-wise ops compute in the stated precision, one rounding per
 *     arithmetic operation (compiled with -ffp-contract=off, no FMA);
 *   - ippsAddProduct_32fc: dst[n] += src1[n] * src2[n] (complex product);
 *   - ippsDivC_32fc_I: complex division by a constant, textbook formula;
 *   - ippsSinCos_32f_A11: sin/cos from libm (IPP's A11 variant is only ~11-bit
 *     accurate, libm is at least that);
 *   - ippsFFTFwd_CToC_32fc: X[k] = sum_n x[n] e^{-2 pi i n k / N}; with
 *     IPP_FFT_NODIV_BY_ANY (used by kernel.c:179,185 via vectordefs.h:61) the
 *     result is not scaled.  Written as an iterative radix-2 decimation-in-time
 *     Cooley-Tukey transform (Cooley & Tukey 1965) with the twiddle table built
 *     in double precision at init and stored as float.
 */
#include "ipps.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SHIM_ALIGN 64

static void* shim_alloc(size_t bytes)
{
    void* p = NULL;
    if (bytes == 0) bytes = 1;
    if (posix_memalign(&p, SHIM_ALIGN, (bytes + SHIM_ALIGN - 1) / SHIM_ALIGN * SHIM_ALIGN) != 0) return NULL;
    return p;
}

Ipp8u*   ippsMalloc_8u(int len)   { return (Ipp8u*)shim_alloc((size_t)len); }
Ipp32f*  ippsMalloc_32f(int len)  { return (Ipp32f*)shim_alloc((size_t)len * sizeof(Ipp32f)); }
Ipp64f*  ippsMalloc_64f(int len)  { return (Ipp64f*)shim_alloc((size_t)len * sizeof(Ipp64f)); }
Ipp32fc* ippsMalloc_32fc(int len) { return (Ipp32fc*)shim_alloc((size_t)len * sizeof(Ipp32fc)); }
Ipp64fc* ippsMalloc_64fc(int len) { return (Ipp64fc*)shim_alloc((size_t)len * sizeof(Ipp64fc)); }
void ippsFree(void* ptr) { free(ptr); }
void ippFree(void* ptr)  { free(ptr); }

#define CHECK_PTR(p) do { if (!(p)) return ippStsNullPtrErr; } while (0)
#define CHECK_LEN(n) do { if ((n) <= 0) return ippStsSizeErr; } while (0)

IppStatus ippsAdd_32fc_I(const Ipp32fc* s, Ipp32fc* sd, int len)
{
    CHECK_PTR(s); CHECK_PTR(sd); CHECK_LEN(len);
    for (int n = 0; n < len; n++) { sd[n].re = sd[n].re + s[n].re; sd[n].im = sd[n].im + s[n].im; }
    return ippStsNoErr;
}

IppStatus ippsAddC_64f_I(Ipp64f val, Ipp64f* sd, int len)
{
    CHECK_PTR(sd); CHECK_LEN(len);
    for (int n = 0; n < len; n++) sd[n] = sd[n] + val;
    return ippStsNoErr;
}

IppStatus ippsAddProduct_32fc(const Ipp32fc* a, const Ipp32fc* b, Ipp32fc* acc, int len)
{
    CHECK_PTR(a); CHECK_PTR(b); CHECK_PTR(acc); CHECK_LEN(len);
    for (int n = 0; n < len; n++) {
        float pr = a[n].re * b[n].re - a[n].im * b[n].im;
        float pi = a[n].re * b[n].im + a[n].im * b[n].re;
        acc[n].re = acc[n].re + pr;
        acc[n].im = acc[n].im + pi;
    }
    return ippStsNoErr;
}

IppStatus ippsConj_32fc(const Ipp32fc* s, Ipp32fc* d, int len)
{
    CHECK_PTR(s); CHECK_PTR(d); CHECK_LEN(len);
    for (int n = 0; n < len; n++) { d[n].re = s[n].re; d[n].im = -s[n].im; }
    return ippStsNoErr;
}

IppStatus ippsDivC_32fc_I(Ipp32fc v, Ipp32fc* sd, int len)
{
    CHECK_PTR(sd); CHECK_LEN(len);
    float den = v.re * v.re + v.im * v.im;
    if (den == 0.0f) return -10; /* ippStsDivByZeroErr */
    for (int n = 0; n < len; n++) {
        float xr = sd[n].re, xi = sd[n].im;
        sd[n].re = (xr * v.re + xi * v.im) / den;
        sd[n].im = (xi * v.re - xr * v.im) / den;
    }
    return ippStsNoErr;
}

IppStatus ippsMagnitude_32fc(const Ipp32fc* s, Ipp32f* d, int len)
{
    CHECK_PTR(s); CHECK_PTR(d); CHECK_LEN(len);
    for (int n = 0; n < len; n++) d[n] = sqrtf(s[n].re * s[n].re + s[n].im * s[n].im);
    return ippStsNoErr;
}

IppStatus ippsMul_32fc(const Ipp32fc* a, const Ipp32fc* b, Ipp32fc* d, int len)
{
    CHECK_PTR(a); CHECK_PTR(b); CHECK_PTR(d); CHECK_LEN(len);
    for (int n = 0; n < len; n++) {
        float r = a[n].re * b[n].re - a[n].im * b[n].im;
        float i = a[n].re * b[n].im + a[n].im * b[n].re;
        d[n].re = r; d[n].im = i;
    }
    return ippStsNoErr;
}

IppStatus ippsMul_32fc_I(const Ipp32fc* s, Ipp32fc* sd, int len)
{
    return ippsMul_32fc(s, sd, sd, len);
}

IppStatus ippsMulC_32f(const Ipp32f* s, Ipp32f val, Ipp32f* d, int len)
{
    CHECK_PTR(s); CHECK_PTR(d); CHECK_LEN(len);
    for (int n = 0; n < len; n++) d[n] = s[n] * val;
    return ippStsNoErr;
}

IppStatus ippsMulC_32fc(const Ipp32fc* s, Ipp32fc v, Ipp32fc* d, int len)
{
    CHECK_PTR(s); CHECK_PTR(d); CHECK_LEN(len);
    for (int n = 0; n < len; n++) {
        float r = s[n].re * v.re - s[n].im * v.im;
        float i = s[n].re * v.im + s[n].im * v.re;
        d[n].re = r; d[n].im = i;
    }
    return ippStsNoErr;
}

IppStatus ippsMulC_32fc_I(Ipp32fc v, Ipp32fc* sd, int len)
{
    return ippsMulC_32fc(sd, v, sd, len);
}

IppStatus ippsMulC_64f(const Ipp64f* s, Ipp64f val, Ipp64f* d, int len)
{
    CHECK_PTR(s); CHECK_PTR(d); CHECK_LEN(len);
    for (int n = 0; n < len; n++) d[n] = s[n] * val;
    return ippStsNoErr;
}

IppStatus ippsMulC_64f_I(Ipp64f val, Ipp64f* sd, int len)
{
    return ippsMulC_64f(sd, val, sd, len);
}

IppStatus ippsPhase_32fc(const Ipp32fc* s, Ipp32f* d, int len)
{
    CHECK_PTR(s); CHECK_PTR(d); CHECK_LEN(len);
    for (int n = 0; n < len; n++) d[n] = atan2f(s[n].im, s[n].re);
    return ippStsNoErr;
}

IppStatus ippsRealToCplx_32f(const Ipp32f* re, const Ipp32f* im, Ipp32fc* d, int len)
{
    CHECK_PTR(d); CHECK_LEN(len);
    for (int n = 0; n < len; n++) { d[n].re = re ? re[n] : 0.0f; d[n].im = im ? im[n] : 0.0f; }
    return ippStsNoErr;
}

IppStatus ippsZero_32fc(Ipp32fc* d, int len)
{
    CHECK_PTR(d); CHECK_LEN(len);
    memset(d, 0, (size_t)len * sizeof(Ipp32fc));
    return ippStsNoErr;
}

IppStatus ippsSinCos_32f_A11(const Ipp32f* s, Ipp32f* sn, Ipp32f* cs, Ipp32s len)
{
    CHECK_PTR(s); CHECK_PTR(sn); CHECK_PTR(cs); CHECK_LEN(len);
    for (int n = 0; n < len; n++) { sn[n] = sinf(s[n]); cs[n] = cosf(s[n]); }
    return ippStsNoErr;
}

/* ------------------------------------------------------------------ FFT --- */

struct IppsFFTSpec_C_32fc {
    int order;
    int n;
    int flag;
    Ipp32fc* tw;      /* tw[k] = e^{-2 pi i k / n}, k < n/2 */
    int* bitrev;      /* bit-reversal permutation of [0, n) */
};

static size_t spec_bytes(int order)
{
    size_t n = (size_t)1 << order;
    return sizeof(struct IppsFFTSpec_C_32fc) + SHIM_ALIGN + (n / 2 + 1) * sizeof(Ipp32fc) + SHIM_ALIGN +
           n * sizeof(int) + SHIM_ALIGN;
}

IppStatus ippsFFTGetSize_C_32fc(int order, int flag, IppHintAlgorithm hint,
                                int* pSpecSize, int* pSpecBufferSize, int* pBufferSize)
{
    (void)flag; (void)hint;
    if (order < 0 || order > 27) return ippStsFftOrderErr;
    CHECK_PTR(pSpecSize); CHECK_PTR(pSpecBufferSize); CHECK_PTR(pBufferSize);
    *pSpecSize = (int)spec_bytes(order);
    *pSpecBufferSize = 64;
    *pBufferSize = (int)(((size_t)1 << order) * sizeof(Ipp32fc));
    return ippStsNoErr;
}

static void* align_up(void* p)
{
    uintptr_t u = (uintptr_t)p;
    return (void*)((u + SHIM_ALIGN - 1) / SHIM_ALIGN * SHIM_ALIGN);
}

IppStatus ippsFFTInit_C_32fc(IppsFFTSpec_C_32fc** ppFFTSpec, int order, int flag,
                             IppHintAlgorithm hint, Ipp8u* pSpec, Ipp8u* pSpecBuffer)
{
    (void)hint; (void)pSpecBuffer;
    CHECK_PTR(ppFFTSpec); CHECK_PTR(pSpec);
    if (order < 0 || order > 27) return ippStsFftOrderErr;
    struct IppsFFTSpec_C_32fc* sp = (struct IppsFFTSpec_C_32fc*)align_up(pSpec);
    int n = 1 << order;
    sp->order = order;
    sp->n = n;
    sp->flag = flag;
    sp->tw = (Ipp32fc*)align_up((Ipp8u*)sp + sizeof(*sp));
    sp->bitrev = (int*)align_up((Ipp8u*)(sp->tw + n / 2 + 1));
    for (int k = 0; k < n / 2 + 1; k++) {
        double ang = -2.0 * IPP_PI * (double)k / (double)n;
        sp->tw[k].re = (float)cos(ang);
        sp->tw[k].im = (float)sin(ang);
    }
    for (int i = 0; i < n; i++) {
        int r = 0;
        for (int b = 0; b < order; b++) r |= ((i >> b) & 1) << (order - 1 - b);
        sp->bitrev[i] = r;
    }
    *ppFFTSpec = sp;
    return ippStsNoErr;
}

IppStatus ippsFFTFwd_CToC_32fc(const Ipp32fc* src, Ipp32fc* dst,
                               const IppsFFTSpec_C_32fc* sp, Ipp8u* pBuffer)
{
    CHECK_PTR(src); CHECK_PTR(dst); CHECK_PTR(sp);
    int n = sp->n;
    Ipp32fc* work = pBuffer ? (Ipp32fc*)pBuffer : dst;
    /* bit-reversed copy (through the work buffer so src == dst is allowed) */
    for (int i = 0; i < n; i++) work[sp->bitrev[i]] = src[i];
    for (int half = 1; half < n; half <<= 1) {
        int step = n / (2 * half);
        for (int base = 0; base < n; base += 2 * half) {
            for (int k = 0; k < half; k++) {
                Ipp32fc w = sp->tw[k * step];
                Ipp32fc a = work[base + k];
                Ipp32fc b = work[base + k + half];
                float tr = b.re * w.re - b.im * w.im;
                float ti = b.re * w.im + b.im * w.re;
                work[base + k].re = a.re + tr;
                work[base + k].im = a.im + ti;
                work[base + k + half].re = a.re - tr;
                work[base + k + half].im = a.im - ti;
            }
        }
    }
    float scale = 1.0f;
    if (sp->flag == IPP_FFT_DIV_FWD_BY_N) scale = 1.0f / (float)n;
    else if (sp->flag == IPP_FFT_DIV_BY_SQRTN) scale = 1.0f / sqrtf((float)n);
    if (work != dst || scale != 1.0f) {
        for (int i = 0; i < n; i++) { dst[i].re = work[i].re * scale; dst[i].im = work[i].im * scale; }
    }
    return ippStsNoErr;
}
