/*
 * ipps.h -- test-infrastructure stand-in for the subset of Intel IPP that the
 * reference FX correlator (kernel.c, main.c) calls.  Oracle only: nothing in the
 * product links this.
 *
 * Intel IPP is not vendored by the reference (kernel.h:13-15 includes <ipps.h>,
 * <ippvm.h>, <ippcore.h>; CMakeLists.txt:55-68 looks for it under
 * /opt/intel/oneapi/ipp/latest, version unpinned).  The names, argument order and
 * meaning below follow IPP's published API so that kernel.c / main.c compile
 * unchanged; every body in ipp_shim.c is written from the documented semantics
 * (element-wise vector maths, a forward unnormalised complex FFT).
 *
 * Entry points used by the reference (via vectordefs.h:23-67 and directly at
 * kernel.c:179-186): ippsMalloc_{8u,32f,64f,32fc,64fc}, ippsFree, ippFree,
 * ippsAdd_32fc_I, ippsAddC_64f_I, ippsAddProduct_32fc, ippsConj_32fc,
 * ippsDivC_32fc_I, ippsMagnitude_32fc, ippsMul_32fc_I, ippsMulC_32f,
 * ippsMulC_32fc, ippsMulC_64f, ippsPhase_32fc, ippsRealToCplx_32f,
 * ippsSinCos_32f_A11, ippsZero_32fc, ippsFFTGetSize_C_32fc, ippsFFTInit_C_32fc,
 * ippsFFTFwd_CToC_32fc.
 */
#ifndef FXORACLE_IPPS_SHIM_H
#define FXORACLE_IPPS_SHIM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef uint8_t  Ipp8u;
typedef int16_t  Ipp16s;
typedef int32_t  Ipp32s;
typedef float    Ipp32f;
typedef double   Ipp64f;
typedef struct { Ipp32f re; Ipp32f im; } Ipp32fc;
typedef struct { Ipp64f re; Ipp64f im; } Ipp64fc;

typedef int IppStatus;
enum { ippStsNoErr = 0, ippStsNullPtrErr = -8, ippStsSizeErr = -6, ippStsFftOrderErr = -15 };

typedef enum { ippAlgHintNone = 0, ippAlgHintFast = 1, ippAlgHintAccurate = 2 } IppHintAlgorithm;

/* FFT normalisation flags (IPP numbering). */
#define IPP_FFT_DIV_FWD_BY_N 1
#define IPP_FFT_DIV_INV_BY_N 2
#define IPP_FFT_DIV_BY_SQRTN 4
#define IPP_FFT_NODIV_BY_ANY 8

#define IPP_PI 3.14159265358979323846

typedef struct IppsFFTSpec_C_32fc IppsFFTSpec_C_32fc;

/* memory */
Ipp8u*   ippsMalloc_8u(int len);
Ipp32f*  ippsMalloc_32f(int len);
Ipp64f*  ippsMalloc_64f(int len);
Ipp32fc* ippsMalloc_32fc(int len);
Ipp64fc* ippsMalloc_64fc(int len);
void     ippsFree(void* ptr);
void     ippFree(void* ptr);

/* element-wise vector maths */
IppStatus ippsAdd_32fc_I(const Ipp32fc* pSrc, Ipp32fc* pSrcDst, int len);
IppStatus ippsAddC_64f_I(Ipp64f val, Ipp64f* pSrcDst, int len);
IppStatus ippsAddProduct_32fc(const Ipp32fc* pSrc1, const Ipp32fc* pSrc2, Ipp32fc* pSrcDst, int len);
IppStatus ippsConj_32fc(const Ipp32fc* pSrc, Ipp32fc* pDst, int len);
IppStatus ippsDivC_32fc_I(Ipp32fc val, Ipp32fc* pSrcDst, int len);
IppStatus ippsMagnitude_32fc(const Ipp32fc* pSrc, Ipp32f* pDst, int len);
IppStatus ippsMul_32fc(const Ipp32fc* pSrc1, const Ipp32fc* pSrc2, Ipp32fc* pDst, int len);
IppStatus ippsMul_32fc_I(const Ipp32fc* pSrc, Ipp32fc* pSrcDst, int len);
IppStatus ippsMulC_32f(const Ipp32f* pSrc, Ipp32f val, Ipp32f* pDst, int len);
IppStatus ippsMulC_32fc(const Ipp32fc* pSrc, Ipp32fc val, Ipp32fc* pDst, int len);
IppStatus ippsMulC_32fc_I(Ipp32fc val, Ipp32fc* pSrcDst, int len);
IppStatus ippsMulC_64f(const Ipp64f* pSrc, Ipp64f val, Ipp64f* pDst, int len);
IppStatus ippsMulC_64f_I(Ipp64f val, Ipp64f* pSrcDst, int len);
IppStatus ippsPhase_32fc(const Ipp32fc* pSrc, Ipp32f* pDst, int len);
IppStatus ippsRealToCplx_32f(const Ipp32f* pSrcRe, const Ipp32f* pSrcIm, Ipp32fc* pDst, int len);
IppStatus ippsZero_32fc(Ipp32fc* pDst, int len);

/* FFT: forward complex-to-complex, e^{-i}, normalisation per flag */
IppStatus ippsFFTGetSize_C_32fc(int order, int flag, IppHintAlgorithm hint,
                                int* pSpecSize, int* pSpecBufferSize, int* pBufferSize);
IppStatus ippsFFTInit_C_32fc(IppsFFTSpec_C_32fc** ppFFTSpec, int order, int flag,
                             IppHintAlgorithm hint, Ipp8u* pSpec, Ipp8u* pSpecBuffer);
IppStatus ippsFFTFwd_CToC_32fc(const Ipp32fc* pSrc, Ipp32fc* pDst,
                               const IppsFFTSpec_C_32fc* pFFTSpec, Ipp8u* pBuffer);

/* ippvm: vector sin/cos (the _A11 accuracy suffix is honoured by using libm) */
IppStatus ippsSinCos_32f_A11(const Ipp32f* pSrc, Ipp32f* pDst1, Ipp32f* pDst2, Ipp32s len);

#ifdef __cplusplus
}
#endif
#endif
