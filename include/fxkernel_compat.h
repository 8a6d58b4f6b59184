/*
 * fxkernel_compat.h -- the reference correlator's kernel.h entry points, served
 * by libfxcorr.so on the GPU.
 *
 * A host written against the reference (main.c) links against libfxcorr.so
 * instead of kernel.c and runs unchanged: same arguments, same visibility
 * arrays, same vis.out.  Declarations match kernel.h (cited per function);
 * cf32 here is layout-identical to the reference's Ipp32fc {float re, im}.
 *
 * Behaviour that differs from kernel.c, by design:
 *   - the unpacked / channelised / conjchannels scratch arrays are allocated as
 *     the reference does but not filled (the GPU keeps its intermediates on the
 *     device);
 *   - errors are reported on stderr and through fxc_compat_last_error(); the
 *     library never calls exit();
 *   - nchan may be any power of two in [128, 4096] (kernel.c:31-35 requires a
 *     perfect square); stridesize is still reported as (int)sqrt(nchan);
 *   - the X stage is FP32 (1e-5 parity with kernel.c); setting the environment
 *     variable FXC_COMPAT_XMODE=tc (or fp8) selects the FP16 (or FP8) tensor-core form;
 *   - single-threaded like the reference (one cached GPU context per process).
 */
#ifndef FXKERNEL_COMPAT_H
#define FXKERNEL_COMPAT_H

#include <time.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef struct { float re; float im; } fxc_cf32;

/* kernel.h:63-66, kernel.c:8-115 */
void init_FxKernel(int* nant, int* nchan, int* nbit, double* lo, double* bw, struct timespec* starttime,
                   char* starttimestring, int* fftchannels, double* sampletime, int* stridesize, int* substridesize,
                   int* fractionalLoFreq, fxc_cf32*** unpacked, fxc_cf32*** channelised, fxc_cf32*** conjchannels,
                   fxc_cf32*** visibilities, int* nbaselines, int* baselineCount, int split);

/* kernel.h:106-110, kernel.c:709-827: accumulates the FFTs iteration[0..numffts-1] (absolute indices; the
 * subintegration holds numffts*split FFTs) into visibilities[b][2l+m][chan] and baselineCount[b]. */
void processAntennasAndBaselinePara(int* nant, int* numffts, int* fftchannels, double* antFileOffsets,
                                    double* sampletime, unsigned char** inputData, fxc_cf32*** unpacked,
                                    fxc_cf32*** channelised, fxc_cf32*** conjchannels, double** delays, int* nbit,
                                    int* substridesize, int* stridesize, int* fractionalLoFreq, double* lo,
                                    int* nchan, fxc_cf32*** visibilities, int* baselineCount, int* iteration,
                                    double* bw, fxc_cf32*** visibilities_out, int* baselineCount_out, int split);

/* kernel.h:123, kernel.c:856-878 */
void merge(int split, int nbaselines, fxc_cf32*** visibilities, int* nant, int* nChan, int* baselineCount,
           fxc_cf32*** visibilities_out, int* baselineCount_out);

/* kernel.h:95, kernel.c:348-359 */
void processNormalize(int* nbaselines, int* baselineCount, fxc_cf32*** visibilities, int* nchan,
                      fxc_cf32*** visibilities_out);

/* kernel.h:112, kernel.c:361-371 */
void resetBeforeProcess(int* nbaselines, fxc_cf32*** visibilities, int* nchan, int* baselineCount, int split);

/* kernel.h:82, kernel.c:570-630: writes ./vis.out in the reference's text format */
void saveVisibilities(int* nbaselines, int* nchan, fxc_cf32*** visibilities, double* bw);

/* kernel.h:84-88, kernel.c:632-667 */
void startTiming(struct timespec* starttime, char* starttimestring);
void saveLog(long long* diff_ms, char* starttimestring);
void endTiming(struct timespec* starttime, long long* diff_ms);

/* FXC_OK or the status of the last failing call above (no counterpart in the reference, which exits). */
int fxc_compat_last_error(void);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
