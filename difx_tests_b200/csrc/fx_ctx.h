// fx_ctx.h -- the correlation context behind the C ABI (internal; shared by
// fx_api.cu and the multi-job batch in fx_batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/fxcorr.h"
#include "fx_internal.h"

struct fxc_ctx {
    fxc_config cfg;
    int device = 0;
    int F = 0, nsig = 0, npair = 0, npair_ant = 0, nbl = 0, nout = 0;
    int ld = 0;            // delay-table leading dimension (FFTs, multiple of 128)
    int T = 0;             // FFT slots per chunk (multiple of 64)
    int nsb_g = 1;         // subbands per chunk (all of them unless the problem is large)
    int rows = 0;          // F16 spectra rows per channel
    size_t pitch = 0;      // input row pitch
    size_t subint = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    uint8_t* d_in = nullptr;
    double* d_delays = nullptr;
    double* d_offs = nullptr;
    double* d_sblo = nullptr;
    float* d_chan_sub = nullptr;
    float* d_chan_step = nullptr;
    fx::DelayEntry* d_dtab = nullptr;
    uint32_t* d_vbits = nullptr;
    void* d_spec = nullptr;
    size_t spec_bytes = 0;
    // F-stage output layout: kSpecF32 [sb][sig][T][chan] (the plain form, and the FP16 tensor-core
    // form of up to 64 signals on the FFT F stage, whose X stage casts to FP16 on the way into the
    // MMA operand: xf32) or kSpecF16 K-major [sb][chan][rows][T] (the other tensor-core forms)
    int spec_mode = 0;
    bool xf32 = false;
    uint8_t* d_spec8 = nullptr;   // FP8 form: e4m3 spectra [nsb][nchan][rows][T]
    unsigned* d_amax = nullptr;   // FP8 form: [nsb*nchan][nsig] absmax bits of the chunk
    float* d_inv = nullptr;       // FP8 form: [nsb*nchan][nsig] inverse scales
    float2* d_acc = nullptr;
    size_t acc_bytes = 0;
    void* d_xpart = nullptr;      // plain form with few channel groups: X-stage segment partial sums
    int xseg_max = 1;             // segments it holds
    int* d_counts = nullptr;
    int* d_err = nullptr;   // device-side wait expiry code of the tensor-core X stage
    int nsm = 148;
    // delay-model upload: [3*nant delays | nant file offsets] (d_delays), or window descriptors
    // [nant bases | nant lengths], through a pinned ring of slots
    static constexpr int NRING = 4;
    static constexpr int NMODEL = 6;   // doubles per antenna in a ring slot
    double* d_win_meta = nullptr;      // NWIN + 1 window descriptors (host windows, caller's rows)
    // streamed host input: two device windows of win_cap samples per row, filled on copy_stream
    int win_ffts = 0;
    long long win_cap = 0;
    size_t win_pitch = 0;
    static constexpr int NWIN = 3;     // copies may run two windows ahead of the correlation
    uint8_t* d_win[NWIN] = {};
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t win_ready[NWIN] = {};
    cudaEvent_t win_free[NWIN] = {};
    int win_next = 0;
    double* h_stage = nullptr;
    cudaEvent_t stage_ev[NRING] = {};
    int stage_next = 0;
    std::vector<double> last_model;
    bool model_valid = false;
    float2* d_vis = nullptr;
    size_t vis_bytes = 0;
    // stage timing (fxc_enable_stage_timing / fxc_stage_times)
    bool timing = false;
    struct Pending {
        int stage;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;
    double stage_ms[FXC_NSTAGE] = {0, 0, 0, 0};
    long long stage_launches[FXC_NSTAGE] = {0, 0, 0, 0};
    // launch plan (fxc_set_plan / fxc_autotune / plan cache): FFTs per F-stage CTA, plain X tile variant
    int plan_tb = 16;
    int plan_alt = 0;
};

// Plan cache (file named by FXC_PLAN_CACHE): lines "<key...> <value>", later lines win.
// Keys: "F <fft> <npol>" FFTs per CTA of the FP32-output F stage, "H <fft> <npol>" of the
// F16-output F stage, "X <signal blocks of 8>" plain X tile variant.
std::map<std::string, int> plan_cache_load();
void plan_cache_append(const std::vector<std::string>& lines);

// fxc_create with control over subband grouping (false: every subband in each chunk, as the
// multi-job batch's task tables assume)
int ctx_create(const fxc_config* cfg, fxc_ctx** out, bool group_subbands);

// delay model to the device (only when it changed) + K0 over FFTs first..first+nfft-1; with a
// device window descriptor d_meta ([nant bases | nant lengths], samples) the input rows are
// windows (see k_delay_table)
int ctx_run_delay_table(fxc_ctx* x, const double* delays, const double* offs, int first, int nfft, int* ld_out,
                        const double* d_meta = nullptr);
// F-stage arguments of this context for device input rows d_data of `pitch` bytes
fx::FArgs ctx_fargs(fxc_ctx* x, const uint8_t* d_data, size_t pitch, int ld);
// the plain X stage's time segments for xa (its nsig and alt set): tseg, tlen, part
void ctx_xsegments(const fxc_ctx* x, fx::XArgs& xa);
