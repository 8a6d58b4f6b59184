/*
 * fxcorr.h -- C ABI of the B200 (sm_100a) FX correlator hot path.
 *
 * Drop-in for the per-subintegration processing of the reference CPU
 * correlator (twiG56/difx_tests, kernel.c): 2-bit unpack, integer and
 * fractional delay, fringe rotation, FFT, fractional-sample correction and
 * baseline cross-multiply-accumulate, on one GPU.  Plain pointers and sizes
 * only; every call returns an int status (FXC_OK or a negative FXC_ERR_*),
 * never exits the process.  One context per host thread; contexts on the same
 * device may run concurrently on different streams.
 *
 * Reference interfaces replaced (file:line in the reference):
 *   init_FxKernel                   kernel.h:63-66, kernel.c:8-115   -> fxc_create
 *   processAntennasAndBaselinePara  kernel.h:106-110, kernel.c:709-827
 *                                                                    -> fxc_process_host / fxc_process_device
 *   merge                           kernel.h:123, kernel.c:856-878   -> accumulation across calls (fxc_process_*)
 *   processNormalize                kernel.h:95, kernel.c:348-359    -> fxc_get_visibilities(normalize = 1)
 *   resetBeforeProcess              kernel.h:112, kernel.c:361-371   -> fxc_reset
 *   allocDataHost (subintbytes)     allocDataHost.c:8-22             -> fxc_subint_bytes
 * The exact reference symbols (init_FxKernel, processAntennasAndBaselinePara,
 * merge, processNormalize, saveVisibilities, ...) are exported by the
 * compatibility layer declared in fxkernel_compat.h.
 */
#ifndef FXCORR_H
#define FXCORR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define FXC_OK                0
#define FXC_ERR_INVALID      -1   /* bad configuration or argument */
#define FXC_ERR_CUDA         -2   /* CUDA runtime error (see fxc_last_cuda_error) */
#define FXC_ERR_NOMEM        -3   /* device or pinned-host allocation failed */
#define FXC_ERR_UNSUPPORTED  -4   /* valid request this library does not implement */
#define FXC_ERR_NODEVICE     -5   /* no sm_100 CUDA device */
#define FXC_ERR_TIMEOUT      -6   /* a bounded device-side wait expired; that call's result is invalid */

/* X-stage arithmetic */
#define FXC_X_PLAIN_FP32 0        /* FP32 CUDA-core cross-multiply-accumulate */
#define FXC_X_TC_FP16    1        /* tcgen05 tensor cores, FP16 inputs, FP32 accumulation (on the FFT F
                                     stage with <= 64 signals the F stage writes FP32 spectra and the X
                                     stage rounds them to FP16 itself; FXC_TC_SPECTRA=f16 in the
                                     environment at context creation keeps the F stage's FP16 layout) */
#define FXC_X_TC_FP8     2        /* tcgen05 tensor cores, FP8-E4M3 inputs scaled per antenna, polarisation and
                                     channel by 448/absmax over each spectra chunk, FP32 accumulation */

typedef struct fxc_config {
    int nant;          /* antennas, >= 2; nant * npol <= 512 */
    int npol;          /* 1, or 2 = the reference's interleaved dual-polarisation format */
    int nchan;         /* channels per subband: power of two in [128, 4096]; FFT length 2*nchan */
    int nbit;          /* bits per sample: 2 (the reference's only unpacker, kernel.c:388-395) */
    int iscomplex;     /* 0: real sampling (kernel.c:15) */
    int numffts;       /* FFTs per subintegration; sets the maximum sample offset (kernel.c:730) */
    int nsubband;      /* independent subbands sharing the antennas' delay model, >= 1 */
    int xmode;         /* FXC_X_PLAIN_FP32, FXC_X_TC_FP16 or FXC_X_TC_FP8 */
    double lo;         /* LO (sky) frequency of subband 0, Hz; |lo| < 2^31 for reference-identical phases */
    double bw;         /* bandwidth per subband, Hz; sampling interval 1/(2 bw) (kernel.c:14) */
    double sb_spacing; /* LO step between consecutive subbands, Hz */
    int chunk_ffts;    /* FFTs per F->X chunk (multiple of 64), 0 = chosen by the library: the
                          spectra of a chunk stay within 16 GiB, or
                          the environment variable FXC_SPECTRA_BUDGET_MB; problems too large for
                          long chunks of every subband are chunked over groups of subbands */
    int window_ffts;   /* FFTs per streamed input window (fxc_process_host*); 0 = the chunk length,
                          at most 1024 (three windows in flight: copies run ahead of the correlation).
                          > 0 also drops the whole-subintegration device input buffer, so the
                          subintegration never has to fit in device memory (fxc_upload_input and
                          fxc_device_input then return FXC_ERR_UNSUPPORTED) */
    int fstage;        /* F-stage arithmetic, FXC_F_* (0 = FXC_F_AUTO) */
} fxc_config;

/* F-stage arithmetic (fxc_config.fstage).  The reference's F stage is an FP32 FFT
 * (kernel.c:499-510, IPP ippsFFTFwd_CToC_32fc); every choice but FXC_F_TC16 keeps FP32
 * accuracy.  The X forms read the F stage's output as FP32 (plain) or cast to FP16 / e4m3
 * (tensor-core forms).
 *   FXC_F_AUTO   FXC_F_FFT32.
 *   FXC_F_FFT32  FP32 radix-16 Stockham FFT on the CUDA cores; every geometry and form.
 *   FXC_F_TC16   FP16 DFT on the tensor cores: the 2048-point FFT as two tcgen05 GEMMs with
 *                FP16 DFT matrices and an FP16 intermediate (three FP16 roundings inside the
 *                F stage, spectra RMS error ~2x the FP32 FFT's after the FP16 cast).  Tensor-core
 *                X forms at 1024 channels, one polarisation, 2-bit real input only
 *                (FXC_ERR_UNSUPPORTED otherwise).
 *   FXC_F_TC32   FP32-grade DFT on the tensor cores: the same two tcgen05 GEMMs with every FP16
 *                operand an error-compensated pair (hi + lo) and three products per GEMM
 *                (hi.hi + lo.hi + hi.lo, FP32 accumulation): spectra within ~2e-7 of max|X|, as
 *                the FP32 FFT.  Every X form at 1024 channels, one polarisation, 2-bit real
 *                input (FXC_ERR_UNSUPPORTED otherwise). */
#define FXC_F_AUTO   0
#define FXC_F_FFT32  1
#define FXC_F_TC16   2
#define FXC_F_TC32   3

typedef struct fxc_ctx fxc_ctx;

/* Initialise a config with the reference's defaults (NPOL 2, NBIT 2, COMPLEX 0,
 * main.c:29-31) and one subband. */
void fxc_config_default(fxc_config* cfg);

/* Bytes of one (subband, antenna) input stream for one subintegration:
 * nchan * 2 * (numffts + 1) * nbit / 8 * npol (allocDataHost.c:21). */
size_t fxc_subint_bytes(const fxc_config* cfg);

/* Number of output baselines (A(A-1)/2 crosses in the reference's order, then
 * A autocorrelations) and the size of one visibility set in complex values:
 * nsubband * (nbl + nant) * npol^2 * nchan. */
int fxc_num_baselines(const fxc_config* cfg);
size_t fxc_vis_count(const fxc_config* cfg);

/* Create a context on the current CUDA device: validates the config, allocates
 * all device buffers, zeroes the accumulators. */
int fxc_create(const fxc_config* cfg, fxc_ctx** out);
void fxc_destroy(fxc_ctx* ctx);

/* Zero visibilities and counts (resetBeforeProcess). */
int fxc_reset(fxc_ctx* ctx);

/* Process FFTs first_fft .. first_fft+nfft-1 (0 <= first_fft, first_fft+nfft <= numffts)
 * and accumulate into the context's visibilities.  Calls accumulate, so time
 * shards of one subintegration may be processed by successive calls (the
 * reference's split/merge, main.c:398-433).  The input streams to the device in
 * windows of window_ffts FFTs whose copies overlap the previous window's
 * correlation (see fxc_process_host_window).
 *   data[sb*nant + ant]  host pointer to the subintegration's packed bytes
 *                        (fxc_subint_bytes each); pinned memory (fxc_host_alloc)
 *                        transfers fastest and lets copies overlap compute
 *   delays[3*ant + k]    (quad, lin, const) seconds, t in FFT units (kernel.c:378-380)
 *   fileoffsets[ant]     seconds (kernel.c:736)
 */
int fxc_process_host(fxc_ctx* ctx, const uint8_t* const* data, const double* delays, const double* fileoffsets,
                     int first_fft, int nfft);

/* Same with the input already in device memory: d_data holds nsubband*nant rows
 * of `pitch` bytes (pitch >= fxc_subint_bytes + 16, multiple of 16, 16-byte
 * aligned base).  delays / fileoffsets are host arrays. */
int fxc_process_device(fxc_ctx* ctx, const uint8_t* d_data, size_t pitch, const double* delays,
                       const double* fileoffsets, int first_fft, int nfft);

/* Copy one subintegration's host input rows (data[sb*nant + ant], fxc_subint_bytes
 * each) into the context's device input buffer, asynchronously on its stream. */
/* Streaming (no counterpart in the reference, whose host reads whole subintegrations,
 * main.c:389-396).  Row r = sb * nant + ant of d_data holds the packed samples of that
 * subband and antenna from subintegration sample base_sample[ant] (a whole byte: a
 * multiple of 4/npol samples) for row_bytes bytes; pitch >= row_bytes + 32, 16-byte
 * aligned.  Correlates FFTs [first, first + nfft).  An FFT that the reference would
 * correlate but whose samples are not all inside its antenna's window is left out and
 * the next synchronising call (fxc_synchronize, fxc_get_visibilities) returns
 * FXC_ERR_INVALID; nothing outside the rows is read. */
int fxc_process_device_window(fxc_ctx* ctx, const uint8_t* d_data, size_t pitch, const long long* base_sample,
                              size_t row_bytes, const double* delays, const double* fileoffsets, int first,
                              int nfft);
/* Host rows of the whole subintegration (as fxc_process_host).  Copies only the bytes
 * FFTs [first, first + nfft) need, window by window (window_ffts FFTs each), into one of
 * three device windows on a copy stream, so the copy of one window overlaps the
 * correlation of the previous one (pinned host rows, e.g. fxc_host_alloc, are needed for
 * the overlap).  fxc_process_host is this call over its FFT range. */
int fxc_process_host_window(fxc_ctx* ctx, const uint8_t* const* data, const double* delays,
                            const double* fileoffsets, int first, int nfft);
int fxc_upload_input(fxc_ctx* ctx, const uint8_t* const* data);

/* The context's own device input buffer (rows of *pitch bytes) for callers
 * that fill device memory themselves. */
int fxc_device_input(fxc_ctx* ctx, uint8_t** d_data, size_t* pitch);

/* Copy visibilities to the host: vis holds fxc_vis_count complex values as
 * interleaved float pairs, layout [sb][bl][2*l + m][chan] with bl = crosses in
 * the reference's order then autos; counts (nbl + nant ints, may be NULL) get
 * the number of FFTs accumulated per baseline.  normalize != 0 divides each
 * baseline by its count (processNormalize, kernel.c:348-359).  vis may be NULL
 * when counts is not: the counts alone (e.g. beside fxc_get_visibilities_device). */
int fxc_get_visibilities(fxc_ctx* ctx, float* vis, int* counts, int normalize);

/* Same into device memory (d_vis: fxc_vis_count complex values). */
int fxc_get_visibilities_device(fxc_ctx* ctx, float* d_vis, int normalize);

/* Amplitude and phase (radians) of every visibility, computed on the device: the
 * layout of fxc_get_visibilities with each (re, im) pair replaced by (|v|,
 * atan2(im, re)), the two columns saveVisibilities prints beside re and im
 * (kernel.c:594-596, vectorMagnitude / vectorPhase). */
int fxc_get_amp_phase(fxc_ctx* ctx, float* ampphase, int normalize);

/* Stream used by the context (a cudaStream_t); NULL restores the context's own. */
int fxc_set_stream(fxc_ctx* ctx, void* stream);
int fxc_synchronize(fxc_ctx* ctx);

/* Pinned host memory for input staging. */
int fxc_host_alloc(void** p, size_t bytes);
int fxc_host_free(void* p);

/* One-shot correlation that allocates no memory.  No counterpart in the
 * reference: it is for callers that cannot call cudaMalloc at the point where
 * they correlate -- real-time paths that must not take the allocator's locks or
 * wait on its latency, and hosts whose device memory another framework reserved
 * up front.  The caller passes the input (device rows as for fxc_process_device,
 * host delay model) and the outputs it owns: d_vis (fxc_vis_count complex values,
 * layout of fxc_get_visibilities) and optionally d_counts (nbl + nant ints).
 * Every intermediate lives in one static device array of
 * FXC_NOALLOC_SCRATCH_BYTES that each GPU loading this library holds until the
 * process exits; a problem whose delay table, accumulators and at least 64 FFT
 * slots of spectra do not fit returns FXC_ERR_INVALID.  Plain FP32 X stage only
 * (FXC_ERR_UNSUPPORTED otherwise).  Work is queued on `stream` (a cudaStream_t,
 * NULL = legacy default stream); the call returns before it completes, so a
 * device wait that runs out is reported in the outputs instead: every
 * visibility NaN and every count -6.  All calls share the array: calls that overlap on the GPU race, so order them (one
 * stream, or events). */
#define FXC_NOALLOC_SCRATCH_BYTES (64u << 20)
int fxc_correlate_noalloc(const fxc_config* cfg, const uint8_t* d_data, size_t pitch, const double* delays,
                          const double* fileoffsets, int first_fft, int nfft, float* d_vis, int* d_counts,
                          int normalize, void* stream);

/* ---- many independent jobs in grouped launches ------------------------------
 * A batch holds jobs of uneven geometry (antennas, polarisations, channels,
 * subbands, subintegration length) and X form (plain FP32 or FP16 tensor cores).
 * fxc_batch_process runs every job's whole subintegration: one persistent
 * F-stage launch per group of jobs sharing FFT length, polarisation count and
 * spectra precision (CTAs stride over a task table of {job, subband, antenna
 * block}), one plain X-stage launch per group of jobs of at most 64 signals
 * sharing an X tile plan (one CTA per {job, subband, channel block} task), and
 * one X launch per other job (FP16
 * tensor-core jobs, plain jobs of more than 64 signals), in rounds when a job
 * needs several spectra chunks.  The first call runs eagerly; later calls replay
 * one CUDA graph of the whole sequence.  FXC_ERR_UNSUPPORTED for the FP8 form,
 * input windows, 8-bit complex input and the tensor-core F stages.
 * No counterpart in the reference (one job per run).
 * fxc_batch_autotune times the FFT block size (8/16/32 FFTs per CTA) of every
 * F group and the tile variant of every X group on the uploaded data, keeps the
 * fastest, and zeroes the accumulators; with the environment variable
 * FXC_PLAN_CACHE naming a file, chosen plans are appended to it and read back by
 * later fxc_batch_create calls. */
typedef struct fxc_batch fxc_batch;
int fxc_batch_create(const fxc_config* cfgs, int njobs, fxc_batch** out);
void fxc_batch_destroy(fxc_batch* b);
/* host rows of job `job` (as fxc_upload_input) */
int fxc_batch_upload(fxc_batch* b, int job, const uint8_t* const* data);
/* delay model of job `job` (as fxc_process_host: delays[3*ant+k], fileoffsets[ant]) */
int fxc_batch_set_model(fxc_batch* b, int job, const double* delays, const double* fileoffsets);
int fxc_batch_process(fxc_batch* b);
int fxc_batch_reset(fxc_batch* b);
int fxc_batch_get_visibilities(fxc_batch* b, int job, float* vis, int* counts, int normalize);
int fxc_batch_autotune(fxc_batch* b, int reps);
/* plan of a job's groups: FFTs per F-stage CTA and X tile variant (0/1) */
int fxc_batch_get_plan(fxc_batch* b, int job, int* fft_block, int* x_variant);
int fxc_batch_set_stream(fxc_batch* b, void* stream);
int fxc_batch_synchronize(fxc_batch* b);
/* 0 disables graph capture (every call runs eagerly), non-zero enables it (default) */
int fxc_batch_use_graph(fxc_batch* b, int enable);
/* kernels one fxc_batch_process call launches (delay tables, counts, grouped F and X launches);
 * builds the task tables if needed; < 0 on error */
int fxc_batch_launch_count(fxc_batch* b);

/* Launch plan of a context: FFTs per F-stage CTA (8, 16 or 32) and plain X tile variant (0 or 1).
 * Defaults 16 / 0, or the entries of the plan-cache file named by the environment variable
 * FXC_PLAN_CACHE when the context is created.  Plans change speed only, never results. */
int fxc_set_plan(fxc_ctx* ctx, int fft_block, int x_variant);
int fxc_get_plan(fxc_ctx* ctx, int* fft_block, int* x_variant);
/* Times every plan on the context's current input and delay model (at least one earlier
 * fxc_process_* call) with `reps` launches each, keeps the fastest, appends it to the plan cache
 * (when FXC_PLAN_CACHE is set) and clears the accumulators as fxc_reset does. */
int fxc_autotune(fxc_ctx* ctx, int reps);

/* Per-stage device timing (the counterpart of the reference's per-stage clock()
 * timers, kernel.c:720-821).  With enable != 0 every launch is bracketed by CUDA
 * events on the context's stream.  fxc_stage_times waits for the stream and
 * returns accumulated milliseconds and launch counts per stage
 * [0] delay table + counts, [1] F stage, [2] X stage, [3] finalise;
 * reset != 0 clears the accumulators.  Launch counts are kept even when timing
 * is disabled. */
#define FXC_NSTAGE 4
int fxc_enable_stage_timing(fxc_ctx* ctx, int enable);
int fxc_stage_times(fxc_ctx* ctx, double* ms, long long* launches, int reset);

const char* fxc_strerror(int status);
/* Last CUDA error code seen by this thread's calls (cudaError_t as int). */
int fxc_last_cuda_error(void);
/* Which device-side wait expired when a call returned FXC_ERR_TIMEOUT on this
 * thread: tensor-core X stage 1 stage load, 2 stage release, 3 accumulator release,
 * 4 accumulator ready, 5 drain at exit; F stage 6 input staging copy, 7 a wait of the
 * tensor-core F stage (input copy, stage ring, TMEM hand-off or drain); 0 if none.
 * (16 after FXC_ERR_INVALID: an FFT's input was outside its window.) */
int fxc_last_device_error(void);

/* ---- inspection entry points (parity tests; not needed for correlation) ---- */

/* Delay table of FFTs first_fft..first_fft+nfft-1 computed on the GPU
 * (kernel.c:733-756): offsets / valid as int [nant][nfft], frac / a / b as
 * double [nant][nfft] (any may be NULL). */
int fxc_debug_delay_table(fxc_ctx* ctx, const double* delays, const double* fileoffsets, int first_fft, int nfft,
                          int* offsets, int* valid, double* frac, double* a, double* b);

/* Unpacked 2-bit samples (before fringe rotation) of the F stage for FFTs
 * first_fft..+nfft-1 from the context's device input buffer:
 * out float [nsb][nant][npol][nfft][2*nchan]; zero where an antenna is invalid. */
int fxc_debug_unpack(fxc_ctx* ctx, const double* delays, const double* fileoffsets, int first_fft, int nfft,
                     float* out);

/* F-stage spectra (after fractional-sample correction) for FFTs
 * first_fft..+nfft-1 (nfft <= chunk length) from the context's device input
 * buffer: out interleaved complex float [nsb][nant*npol][nfft][nchan]. */
int fxc_debug_spectra(fxc_ctx* ctx, const double* delays, const double* fileoffsets, int first_fft, int nfft,
                      float* out);

/* Launches a kernel whose bounded device wait (the F stage's input-staging wait, on a
 * barrier that nothing completes) runs out after about 1 s; the next synchronising call
 * returns FXC_ERR_TIMEOUT and fxc_last_device_error() gives 6.  Exercises the failure
 * path of the device waits without faulting the GPU; the context stays usable. */
int fxc_debug_expire_wait(fxc_ctx* ctx);

/* As fxc_debug_expire_wait, for the bounded wait of the tensor-core kernels (the mbarrier
 * wait that the tensor-core F and X stages use for their stage rings and TMEM hand-offs):
 * the next synchronising call returns FXC_ERR_TIMEOUT and fxc_last_device_error() gives 7. */
int fxc_debug_expire_wait_tc(fxc_ctx* ctx);

/* The plain X stage's time-segment cut (up to 64 signals) for `ctas` CTAs of channel groups,
 * `slots` resident CTA slots (SMs x CTAs of the kernel per SM) and T FFT slots per chunk:
 * *tseg segments of *tlen slots (1 and T: no cut).  Host arithmetic only; the library takes
 * the occupancy of its default tile variant on the context's GPU for `slots`. */
int fxc_debug_xplain_segments(long long ctas, long long slots, int T, int* tseg, int* tlen);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
