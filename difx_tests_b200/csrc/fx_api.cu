// fx_api.cu -- C ABI (include/fxcorr.h): context lifetime, buffer layout and
// the per-call launch sequence  K0 delay table -> counts -> [F stage -> X stage]
// per chunk of FFTs -> finalise on demand.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/fxcorr.h"
#include "fx_ctx.h"
#include "fx_internal.h"
#include "fx_kernels.h"

using namespace fx;


namespace {

cudaEvent_t pool_event(fxc_ctx* x)
{
    if (!x->event_pool.empty()) {
        cudaEvent_t e = x->event_pool.back();
        x->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Brackets the launches of one stage with events when timing is enabled.
struct StageScope {
    fxc_ctx* x;
    int stage;
    cudaEvent_t a = nullptr;
    StageScope(fxc_ctx* x_, int s, int nlaunch) : x(x_), stage(s)
    {
        x->stage_launches[s] += nlaunch;
        if (x->timing) {
            a = pool_event(x);
            cudaEventRecord(a, x->stream);
        }
    }
    ~StageScope()
    {
        if (a) {
            cudaEvent_t b = pool_event(x);
            cudaEventRecord(b, x->stream);
            x->pending.push_back({stage, a, b});
        }
    }
};

}  // namespace

static thread_local int g_last_cuda = 0;
static thread_local int g_last_device = 0;

#define FXC_CK(call)                                   \
    do {                                               \
        cudaError_t e_ = (call);                       \
        if (e_ != cudaSuccess) {                       \
            g_last_cuda = (int)e_;                     \
            return e_ == cudaErrorMemoryAllocation ? FXC_ERR_NOMEM : FXC_ERR_CUDA; \
        }                                              \
    } while (0)

static size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

extern "C" {

void fxc_config_default(fxc_config* c)
{
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->npol = 2;
    c->nbit = 2;
    c->iscomplex = 0;
    c->nsubband = 1;
    c->xmode = FXC_X_PLAIN_FP32;
}

size_t fxc_subint_bytes(const fxc_config* c)
{
    if (!c) return 0;
    // allocDataHost.c:21 (cfactor = 2 for real data)
    if (c->iscomplex)   // 8-bit complex: (re, im) bytes per sample and polarisation, nchan samples per FFT
        return (size_t)c->nchan * (size_t)(c->numffts + 1) * 2 * c->npol;
    return (size_t)c->nchan * 2 * (size_t)(c->numffts + 1) * c->nbit / 8 * c->npol;
}

int fxc_num_baselines(const fxc_config* c) { return c ? c->nant * (c->nant - 1) / 2 : 0; }

size_t fxc_vis_count(const fxc_config* c)
{
    if (!c) return 0;
    return (size_t)c->nsubband * (fxc_num_baselines(c) + c->nant) * c->npol * c->npol * c->nchan;
}

const char* fxc_strerror(int s)
{
    switch (s) {
    case FXC_OK: return "ok";
    case FXC_ERR_INVALID: return "invalid configuration or argument";
    case FXC_ERR_CUDA: return "CUDA runtime error";
    case FXC_ERR_NOMEM: return "out of device or pinned host memory";
    case FXC_ERR_UNSUPPORTED: return "not supported by this library";
    case FXC_ERR_NODEVICE: return "no sm_100 CUDA device";
    case FXC_ERR_TIMEOUT: return "device-side wait expired (result invalid)";
    default: return "unknown status";
    }
}

int fxc_last_cuda_error(void) { return g_last_cuda; }
int fxc_last_device_error(void) { return g_last_device; }

static int validate(const fxc_config* c)
{
    if (!c) return FXC_ERR_INVALID;
    if (c->nant < 2 || c->npol < 1 || c->npol > 2 || c->numffts < 1 || c->nsubband < 1) return FXC_ERR_INVALID;
    if (c->nchan < 128 || c->nchan > 4096 || (c->nchan & (c->nchan - 1))) return FXC_ERR_INVALID;
    // 2-bit real (the reference's CPU format) or 8-bit complex (its GPU format, gkernel.cu:277-296)
    if (!((c->nbit == 2 && c->iscomplex == 0) || (c->nbit == 8 && c->iscomplex == 1))) return FXC_ERR_UNSUPPORTED;
    if (c->iscomplex && c->nchan < 256) return FXC_ERR_UNSUPPORTED;   // complex FFT length nchan >= 256
    if (c->iscomplex && (long long)(c->numffts + 1) * c->nchan * 2 * c->npol > 0x7fffffffLL) return FXC_ERR_INVALID;
    if (!(c->bw > 0.0) || !std::isfinite(c->lo) || !std::isfinite(c->sb_spacing)) return FXC_ERR_INVALID;
    if (c->xmode != FXC_X_PLAIN_FP32 && c->xmode != FXC_X_TC_FP16 && c->xmode != FXC_X_TC_FP8)
        return FXC_ERR_INVALID;
    if (c->chunk_ffts < 0 || c->chunk_ffts % (c->xmode == FXC_X_TC_FP8 ? 128 : 64)) return FXC_ERR_INVALID;
    if (c->window_ffts < 0) return FXC_ERR_INVALID;
    if ((long long)(c->numffts + 1) * 2 * c->nchan > 0x7fffffffLL) return FXC_ERR_INVALID;  // int sample offsets
    // plain X: 8x8 register tiles, one CTA per channel group (<= 64 signals) or per pair of
    // 64-signal super-blocks; tensor-core X: 128x128 block pairs of the Gram
    if (c->nant * c->npol > 512) return FXC_ERR_UNSUPPORTED;
    if (c->fstage < FXC_F_AUTO || c->fstage > FXC_F_TC32) return FXC_ERR_INVALID;
    if (c->fstage == FXC_F_TC16 &&
        !(c->xmode != FXC_X_PLAIN_FP32 && c->nchan == 1024 && c->npol == 1 && !c->iscomplex))
        return FXC_ERR_UNSUPPORTED;
    if (c->fstage == FXC_F_TC32 && !(c->nchan == 1024 && c->npol == 1 && !c->iscomplex)) return FXC_ERR_UNSUPPORTED;
    return FXC_OK;
}

}  // extern "C"

std::map<std::string, int> plan_cache_load()
{
    std::map<std::string, int> m;
    const char* path = std::getenv("FXC_PLAN_CACHE");
    if (!path) return m;
    FILE* f = std::fopen(path, "r");
    if (!f) return m;
    char line[256];
    while (std::fgets(line, sizeof line, f)) {
        std::string l(line);
        while (!l.empty() && (l.back() == '\n' || l.back() == '\r' || l.back() == ' ')) l.pop_back();
        const size_t sp = l.rfind(' ');
        if (sp == std::string::npos || sp == 0) continue;
        char* end = nullptr;
        const long v = std::strtol(l.c_str() + sp + 1, &end, 10);
        if (end && *end == '\0') m[l.substr(0, sp)] = (int)v;
    }
    std::fclose(f);
    return m;
}

void plan_cache_append(const std::vector<std::string>& lines)
{
    const char* path = std::getenv("FXC_PLAN_CACHE");
    if (!path) return;
    if (FILE* f = std::fopen(path, "a")) {
        for (const auto& l : lines) std::fprintf(f, "%s\n", l.c_str());
        std::fclose(f);
    }
}

static std::string fplan_key(const fxc_config& c)
{
    return std::string(c.xmode == FXC_X_PLAIN_FP32 ? "F" : "H") + (c.iscomplex ? "C " : " ") +
           std::to_string(c.iscomplex ? c.nchan : 2 * c.nchan) + " " + std::to_string(c.npol);
}

// Input sample geometry: bits per time sample of one row (all polarisations), samples per
// whole byte (window bases are multiples), and the samples of read-ahead past an FFT's last
// sample (the 2-bit unpacker's extra byte, kernel.c:402-409).
static int sample_bits(const fxc_config& c) { return c.iscomplex ? 16 * c.npol : 2 * c.npol; }
static int sample_align(const fxc_config& c) { return std::max(1, 8 / sample_bits(c)); }
static int tail_samples(const fxc_config& c) { return c.iscomplex ? 0 : 8 / sample_bits(c); }
static long long samples_to_bytes(const fxc_config& c, long long s) { return s * sample_bits(c) / 8; }

static std::string xplan_key(int nsig) { return "X " + std::to_string((nsig + 7) / 8); }

extern "C" {

static void free_ctx(fxc_ctx* x)
{
    if (!x) return;
    cudaFree(x->d_in);
    cudaFree(x->d_delays);
    cudaFree(x->d_win_meta);
    for (int s = 0; s < fxc_ctx::NWIN; s++) {
        cudaFree(x->d_win[s]);
        if (x->win_ready[s]) cudaEventDestroy(x->win_ready[s]);
        if (x->win_free[s]) cudaEventDestroy(x->win_free[s]);
    }
    if (x->copy_stream) cudaStreamDestroy(x->copy_stream);
    for (auto& ev : x->stage_ev)
        if (ev) cudaEventDestroy(ev);
    if (x->h_stage) cudaFreeHost(x->h_stage);
    cudaFree(x->d_sblo);
    cudaFree(x->d_chan_sub);
    cudaFree(x->d_chan_step);
    cudaFree(x->d_dtab);
    cudaFree(x->d_vbits);
    cudaFree(x->d_spec);
    cudaFree(x->d_spec8);
    cudaFree(x->d_amax);
    cudaFree(x->d_inv);
    cudaFree(x->d_acc);
    cudaFree(x->d_xpart);
    cudaFree(x->d_counts);
    cudaFree(x->d_err);
    cudaFree(x->d_vis);
    for (auto& p : x->pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (auto e : x->event_pool) cudaEventDestroy(e);
    if (x->own_stream) cudaStreamDestroy(x->own_stream);
    delete x;
}

}  // extern "C"

int ctx_create(const fxc_config* cfg, fxc_ctx** out, bool group_subbands)
{
    if (!out) return FXC_ERR_INVALID;
    *out = nullptr;
    int st = validate(cfg);
    if (st != FXC_OK) return st;
    int dev = 0;
    FXC_CK(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    FXC_CK(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10) return FXC_ERR_NODEVICE;

    fxc_ctx* x = new fxc_ctx();
    x->cfg = *cfg;
    x->device = dev;
    x->nsm = prop.multiProcessorCount;
    const fxc_config& c = x->cfg;
    x->F = c.iscomplex ? c.nchan : 2 * c.nchan;   // complex samples: every FFT bin is a channel
    x->nsig = c.nant * c.npol;
    x->npair = x->nsig * (x->nsig + 1) / 2;
    x->npair_ant = c.nant * (c.nant + 1) / 2;
    x->nbl = c.nant * (c.nant - 1) / 2;
    x->nout = x->nbl + c.nant;
    x->ld = (int)round_up((size_t)c.numffts, 128);
    x->subint = fxc_subint_bytes(cfg);
    x->pitch = round_up(x->subint + 16, 256);
    x->rows = (int)round_up((size_t)2 * x->nsig, 128);

    // Spectra chunk: T FFT slots of nsb_g subbands within a budget of 16 GiB, or
    // FXC_SPECTRA_BUDGET_MB.  Every subband goes into one chunk while that leaves >= 512 slots (or the
    // whole call); larger problems take the subbands in groups so the chunk stays long: both X
    // stages add each chunk's sums to the accumulators once per CTA, so short chunks make them
    // bound by those additions and by each CTA's pipeline fill (the plain X stage at 64 signals
    // x 1024 channels x 8 subbands: 40.9 TFLOP/s at 2 GiB = 504 slots, 48.4 at 16 GiB).
    // Bytes per FFT slot and subband: f32x2 [sb][sig][T][chan] (plain, and the FP16 tensor-core
    // form of up to 64 signals on the FFT F stage: its X stage casts while loading); otherwise
    // f16 [sb][chan][rows][T] (the FP8 form adds an e4m3 copy of half that size; its chunk is a
    // multiple of 128 FFTs).  The F stage's FP32 stores are channel-contiguous, its FP16 K-major
    // stores a corner turn through shared memory per block of FFTs (2048 points, 1 pol: 107 against
    // 90 ms per cfg2 step; 4096 points, 2 pol: 61 against 47 ms per cfg1 step).
    // FXC_TC_SPECTRA=f16 keeps the FP16 layout for every tensor-core form (comparisons).
    const bool tc = c.xmode != FXC_X_PLAIN_FP32;
    const bool fp8 = c.xmode == FXC_X_TC_FP8;
    {
        const char* ts = std::getenv("FXC_TC_SPECTRA");
        const bool force16 = ts && std::strcmp(ts, "f16") == 0;
        x->xf32 = c.xmode == FXC_X_TC_FP16 && (c.fstage == FXC_F_AUTO || c.fstage == FXC_F_FFT32) && x->nsig <= 64 &&
                  c.nchan % 4 == 0 && !force16;
        x->spec_mode = (tc && !x->xf32) ? kSpecF16 : kSpecF32;
    }
    const size_t tq = fp8 ? 128 : 64;
    const size_t per_sb = x->spec_mode == kSpecF16 ? (size_t)c.nchan * x->rows * sizeof(uint16_t)
                                                   : (size_t)x->nsig * c.nchan * sizeof(float2);
    size_t budget = (size_t)16 << 30;
    if (const char* mb = std::getenv("FXC_SPECTRA_BUDGET_MB")) {   // operator override of the budget
        const long long v = std::atoll(mb);
        if (v > 0) budget = (size_t)v << 20;
    }
    const size_t tmax = round_up((size_t)c.numffts, tq);
    const size_t nsb = (size_t)c.nsubband;
    auto fit = [&](size_t bytes_per_slot) { return budget / bytes_per_slot / tq * tq; };
    size_t T, G = nsb;
    if (c.chunk_ffts) {
        T = std::min((size_t)c.chunk_ffts, tmax);
        if (group_subbands) G = std::max<size_t>(1, std::min(nsb, budget / (per_sb * T)));
    } else {
        T = std::min({fit(per_sb * nsb), (size_t)4096, tmax});
        if (group_subbands && T < std::min((size_t)512, tmax)) {
            T = std::min((size_t)2048, tmax);
            G = std::min(nsb, budget / (per_sb * T));
            if (G == 0) {
                G = 1;
                T = std::min(tmax, fit(per_sb));
            }
        }
        if (T < tq) T = tq;
    }
    x->T = (int)T;
    x->nsb_g = (int)G;
    x->spec_bytes = per_sb * G * T;

    auto fail = [&](cudaError_t e) {
        g_last_cuda = (int)e;
        free_ctx(x);
        return e == cudaErrorMemoryAllocation ? FXC_ERR_NOMEM : FXC_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&x->own_stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
    x->stream = x->own_stream;
    const size_t in_bytes = (size_t)c.nsubband * c.nant * x->pitch;
    x->acc_bytes = (size_t)c.nsubband * x->npair * c.nchan * sizeof(float2);
    x->vis_bytes = fxc_vis_count(cfg) * sizeof(float2) / c.nsubband;   // one subband (finalised in turn)
    const int stride = 1 << ((int)std::log2((double)c.nchan) / 2);
    if (c.window_ffts == 0) {   // whole-subintegration device input (fxc_upload_input / fxc_device_input)
        if ((e = cudaMalloc(&x->d_in, in_bytes)) != cudaSuccess) return fail(e);
        if ((e = cudaMemset(x->d_in, 0, in_bytes)) != cudaSuccess) return fail(e);
    }
    // streamed windows: short, so the first copy and the last window's correlation (the parts
    // that cannot overlap) stay small
    x->win_ffts = c.window_ffts > 0 ? c.window_ffts : std::min(x->T, 1024);
    if ((e = cudaMalloc(&x->d_delays, fxc_ctx::NMODEL * sizeof(double) * c.nant)) != cudaSuccess) return fail(e);
    x->d_offs = x->d_delays + 3 * c.nant;
    if ((e = cudaMalloc(&x->d_win_meta, (fxc_ctx::NWIN + 1) * 2 * sizeof(double) * c.nant)) != cudaSuccess)
        return fail(e);
    x->last_model.assign(4 * (size_t)c.nant, 0.0);
    if ((e = cudaHostAlloc(&x->h_stage, fxc_ctx::NRING * fxc_ctx::NMODEL * sizeof(double) * c.nant,
                           cudaHostAllocDefault)) != cudaSuccess)
        return fail(e);
    for (auto& ev : x->stage_ev)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&x->d_sblo, sizeof(double) * c.nsubband)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&x->d_chan_sub, sizeof(float) * stride)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&x->d_chan_step, sizeof(float) * (c.nchan / stride))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&x->d_dtab, sizeof(DelayEntry) * (size_t)c.nant * x->ld)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&x->d_vbits, sizeof(uint32_t) * (size_t)c.nant * (x->ld / 32))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&x->d_spec, x->spec_bytes)) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(x->d_spec, 0, x->spec_bytes)) != cudaSuccess) return fail(e);
    if (fp8) {
        const size_t n8 = x->spec_bytes / 2, nsc = (size_t)x->nsb_g * c.nchan * x->nsig;
        if ((e = cudaMalloc(&x->d_spec8, n8)) != cudaSuccess) return fail(e);
        if ((e = cudaMemset(x->d_spec8, 0, n8)) != cudaSuccess) return fail(e);   // padding rows stay zero
        if ((e = cudaMalloc(&x->d_amax, nsc * sizeof(unsigned))) != cudaSuccess) return fail(e);
        if ((e = cudaMalloc(&x->d_inv, nsc * sizeof(float))) != cudaSuccess) return fail(e);
    }
    if ((e = cudaMalloc(&x->d_acc, x->acc_bytes)) != cudaSuccess) return fail(e);
    if (c.xmode == FXC_X_PLAIN_FP32) {
        // segment partials of the plain X stage when its channel groups underfill the SMs
        int tl = 0;
        xplain_segments(x->nsig, c.nchan, c.nsubband, x->T, x->nsm, &x->xseg_max, &tl);
        if (x->xseg_max > 1 &&
            (e = cudaMalloc(&x->d_xpart, (size_t)x->xseg_max * x->nsb_g * x->npair * c.nchan * sizeof(float2))) !=
                cudaSuccess)
            return fail(e);
    }
    if ((e = cudaMalloc(&x->d_counts, sizeof(int) * x->npair_ant)) != cudaSuccess) return fail(e);
    // d_err[0]: tensor-core X wait-expiry code; d_err[1]: input-window misses
    if ((e = cudaMalloc(&x->d_err, 2 * sizeof(int))) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(x->d_err, 0, 2 * sizeof(int))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&x->d_vis, x->vis_bytes)) != cudaSuccess) return fail(e);

    // constant tables: per-subband LO, f32 channel angular frequencies (kernel.c:162-166)
    std::vector<double> sblo(c.nsubband);
    for (int s = 0; s < c.nsubband; s++) sblo[s] = c.lo + c.sb_spacing * s;
    std::vector<float> csub(stride), cstep(c.nchan / stride);
    const double two_pi = 2 * 3.14159265358979323846;
    for (int j = 0; j < stride; j++) csub[j] = (float)((two_pi * j * c.bw) / (double)c.nchan);
    for (int i = 0; i < c.nchan / stride; i++) cstep[i] = (float)((two_pi * i * stride * c.bw) / (double)c.nchan);
    if ((e = cudaMemcpy(x->d_sblo, sblo.data(), sizeof(double) * c.nsubband, cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e);
    if ((e = cudaMemcpy(x->d_chan_sub, csub.data(), sizeof(float) * stride, cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e);
    if ((e = cudaMemcpy(x->d_chan_step, cstep.data(), sizeof(float) * cstep.size(), cudaMemcpyHostToDevice)) !=
        cudaSuccess)
        return fail(e);
    if ((e = cudaMemset(x->d_acc, 0, x->acc_bytes)) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(x->d_counts, 0, sizeof(int) * x->npair_ant)) != cudaSuccess) return fail(e);
    {
        const auto plans = plan_cache_load();
        auto it = plans.find(fplan_key(c));
        if (it != plans.end() && (it->second == 8 || it->second == 16 || it->second == 32)) x->plan_tb = it->second;
        it = plans.find(xplan_key(x->nsig));
        if (it != plans.end() && (it->second == 0 || it->second == 1)) x->plan_alt = it->second;
    }
    *out = x;
    return FXC_OK;
}

extern "C" {

int fxc_create(const fxc_config* cfg, fxc_ctx** out) { return ctx_create(cfg, out, true); }

void fxc_destroy(fxc_ctx* x)
{
    if (!x) return;
    cudaSetDevice(x->device);
    if (x->stream) cudaStreamSynchronize(x->stream);
    free_ctx(x);
}

int fxc_reset(fxc_ctx* x)
{
    if (!x) return FXC_ERR_INVALID;
    FXC_CK(cudaSetDevice(x->device));
    FXC_CK(cudaMemsetAsync(x->d_acc, 0, x->acc_bytes, x->stream));
    FXC_CK(cudaMemsetAsync(x->d_counts, 0, sizeof(int) * x->npair_ant, x->stream));
    return FXC_OK;
}

int fxc_set_stream(fxc_ctx* x, void* s)
{
    if (!x) return FXC_ERR_INVALID;
    x->stream = s ? (cudaStream_t)s : x->own_stream;
    return FXC_OK;
}

// Reads (and clears) the device-side wait-expiry code; the stream must be idle.
static int device_status(fxc_ctx* x)
{
    int h[2] = {0, 0};
    FXC_CK(cudaMemcpy(h, x->d_err, 2 * sizeof(int), cudaMemcpyDeviceToHost));
    if (h[0] != 0 || h[1] != 0) {
        FXC_CK(cudaMemset(x->d_err, 0, 2 * sizeof(int)));
        g_last_device = h[0] != 0 ? h[0] : h[1];
        return h[0] != 0 ? FXC_ERR_TIMEOUT : FXC_ERR_INVALID;
    }
    return FXC_OK;
}

int fxc_synchronize(fxc_ctx* x)
{
    if (!x) return FXC_ERR_INVALID;
    FXC_CK(cudaSetDevice(x->device));
    FXC_CK(cudaStreamSynchronize(x->stream));
    return device_status(x);
}

int fxc_device_input(fxc_ctx* x, uint8_t** d, size_t* pitch)
{
    if (!x || !d || !pitch) return FXC_ERR_INVALID;
    if (!x->d_in) return FXC_ERR_UNSUPPORTED;
    *d = x->d_in;
    *pitch = x->pitch;
    return FXC_OK;
}

int fxc_host_alloc(void** p, size_t bytes)
{
    if (!p) return FXC_ERR_INVALID;
    FXC_CK(cudaHostAlloc(p, bytes, cudaHostAllocDefault));
    return FXC_OK;
}

int fxc_host_free(void* p)
{
    FXC_CK(cudaFreeHost(p));
    return FXC_OK;
}

}  // extern "C"

// delays / offsets to the device, then K0 over FFTs first..first+nfft-1
// Window bases and lengths (samples; exact as doubles below 2^53) to the device window
// descriptor d_meta, through a pinned ring slot, on stream st.
static int upload_window_meta(fxc_ctx* x, const long long* base, const long long* len, double* d_meta,
                              cudaStream_t st)
{
    const int n = x->cfg.nant;
    const int slot = x->stage_next;
    x->stage_next = (slot + 1) % fxc_ctx::NRING;
    FXC_CK(cudaEventSynchronize(x->stage_ev[slot]));
    double* h = x->h_stage + slot * fxc_ctx::NMODEL * (size_t)n;
    for (int a = 0; a < n; a++) {
        h[a] = (double)base[a];
        h[n + a] = (double)len[a];
    }
    FXC_CK(cudaMemcpyAsync(d_meta, h, 2 * sizeof(double) * n, cudaMemcpyHostToDevice, st));
    FXC_CK(cudaEventRecord(x->stage_ev[slot], st));
    return FXC_OK;
}

int ctx_run_delay_table(fxc_ctx* x, const double* delays, const double* offs, int first, int nfft, int* ld_out,
                        const double* d_meta)
{
    const fxc_config& c = x->cfg;
    if (!delays || !offs || first < 0 || nfft < 1 || (long long)first + nfft > c.numffts) return FXC_ERR_INVALID;
    for (int a = 0; a < 3 * c.nant; a++)
        if (!std::isfinite(delays[a])) return FXC_ERR_INVALID;
    for (int a = 0; a < c.nant; a++)
        if (!std::isfinite(offs[a])) return FXC_ERR_INVALID;
    // The delay model goes to the device only when it changed, through a ring of
    // pinned slots so the copy stays asynchronous (a pageable source would block
    // the host until the stream's earlier work had finished).
    const size_t nmodel = 4 * (size_t)c.nant;
    const size_t slot_doubles = fxc_ctx::NMODEL * (size_t)c.nant;
    bool same = x->model_valid;
    for (size_t i = 0; same && i < 3 * (size_t)c.nant; i++) same = x->last_model[i] == delays[i];
    for (int i = 0; same && i < c.nant; i++) same = x->last_model[3 * c.nant + i] == offs[i];
    if (!same) {
        const int slot = x->stage_next;
        x->stage_next = (slot + 1) % fxc_ctx::NRING;
        FXC_CK(cudaEventSynchronize(x->stage_ev[slot]));
        double* h = x->h_stage + slot * slot_doubles;
        std::memcpy(h, delays, 3 * sizeof(double) * c.nant);
        std::memcpy(h + 3 * c.nant, offs, sizeof(double) * c.nant);
        FXC_CK(cudaMemcpyAsync(x->d_delays, h, nmodel * sizeof(double), cudaMemcpyHostToDevice, x->stream));
        FXC_CK(cudaEventRecord(x->stage_ev[slot], x->stream));
        std::memcpy(x->last_model.data(), h, nmodel * sizeof(double));
        x->model_valid = true;
    }
    const int ld = (int)round_up((size_t)nfft, 128);
    const int maxoffset = (c.numffts - 1) * x->F;  // kernel.c:730
    // kernel.c:14 (real sampling); complex sampling at bw (main_gpu.cu:246-247)
    const double sampletime = c.iscomplex ? 1.0 / c.bw : 1.0 / (2.0 * c.bw);
    FXC_CK(launch_delay_table_window(x->d_delays, x->d_offs, nullptr, first, c.nant, nfft, ld, x->F, maxoffset,
                                     sampletime, d_meta, tail_samples(c), x->d_err + 1,
                                     x->d_dtab, x->d_vbits, x->stream));
    *ld_out = ld;
    return FXC_OK;
}

FArgs ctx_fargs(fxc_ctx* x, const uint8_t* d_data, size_t pitch, int ld)
{
    FArgs a;
    std::memset(&a, 0, sizeof(a));
    a.data = d_data;
    a.pitch = pitch;
    a.dtab = x->d_dtab;
    a.ld = ld;
    a.nant = x->cfg.nant;
    a.npol = x->cfg.npol;
    a.nsb = x->cfg.nsubband;
    a.sb_lo = x->d_sblo;
    a.chan_sub = x->d_chan_sub;
    a.chan_step = x->d_chan_step;
    a.spec = x->d_spec;
    a.rows = x->rows;
    a.T = x->T;
    a.tb = x->plan_tb;
    a.cpx = x->cfg.iscomplex;
    a.err = x->d_err;
    a.fkind = x->cfg.fstage == FXC_F_AUTO ? FXC_F_FFT32 : x->cfg.fstage;
    return a;
}

extern "C" {

}  // extern "C"

extern "C" int fxc_debug_xplain_segments(long long ctas, long long slots, int T, int* tseg, int* tlen)
{
    if (!tseg || !tlen || T < 0) return FXC_ERR_INVALID;
    xplain_segment_model(ctas, slots, T, tseg, tlen);
    return FXC_OK;
}

// The plain X stage's time segments of this context and tile variant (fx_xplain.cu)
void ctx_xsegments(const fxc_ctx* x, XArgs& xa)
{
    xa.tseg = 1;
    xa.tlen = x->T;
    xa.part = nullptr;
    if (!x->d_xpart || xa.nsig > 64) return;
    xplain_segments(xa.nsig, x->cfg.nchan, x->cfg.nsubband, x->T, x->nsm, &xa.tseg, &xa.tlen);
    xa.part = xa.tseg > 1 ? x->d_xpart : nullptr;
}

// One call's correlation of device rows: whole subintegrations (win_base null) or windows.
static int ctx_correlate(fxc_ctx* x, const uint8_t* d_data, size_t pitch, const double* d_meta,
                         const double* delays, const double* offs, int first, int nfft)
{
    int ld = 0;
    {
        StageScope sc(x, 0, 2);
        int st = ctx_run_delay_table(x, delays, offs, first, nfft, &ld, d_meta);
        if (st != FXC_OK) return st;
        FXC_CK(launch_counts(x->d_vbits, x->cfg.nant, ld / 32, x->d_counts, x->stream));
    }
    const bool tc = x->cfg.xmode != FXC_X_PLAIN_FP32;
    const bool fp8 = x->cfg.xmode == FXC_X_TC_FP8;
    FArgs fa = ctx_fargs(x, d_data, pitch, ld);
    fa.amax = x->d_amax;
    XArgs xa{};
    xa.spec = x->d_spec;
    xa.acc = x->d_acc;
    xa.nsig = x->nsig;
    xa.T = x->T;
    xa.nchan = x->cfg.nchan;
    xa.nsb = x->cfg.nsubband;
    xa.rows = x->rows;
    xa.alt = x->plan_alt;
    ctx_xsegments(x, xa);
    const int nsb = x->cfg.nsubband, G = x->nsb_g;
    const FArgs fall = fa;
    const XArgs xall = xa;
    for (int g0 = 0; g0 < nsb; g0 += G)   // subband groups (one group unless the problem is large)
    for (int c0 = 0; c0 < nfft; c0 += x->T) {
        fa = fall;
        xa = xall;
        fa.data = d_data + (size_t)g0 * x->cfg.nant * pitch;
        fa.sb_lo = x->d_sblo + g0;
        fa.nsb = std::min(G, nsb - g0);
        xa.acc = reinterpret_cast<float2*>(x->d_acc) + (size_t)g0 * x->npair * x->cfg.nchan;
        xa.nsb = fa.nsb;
        fa.t_base = c0;
        fa.nfft = std::min(x->T, nfft - c0);
        // slots the chunk uses: the FFTs rounded up to the X stage's stage depth (the F stage
        // writes zeros after the last FFT; later slots keep an earlier chunk's data, unread)
        const int q = fp8 ? 128 : 64;
        fa.tspan = std::min(x->T, (fa.nfft + q - 1) / q * q);
        xa.ntk = fa.tspan;
        {
            StageScope sc(x, 1, 1);
            if (fp8) FXC_CK(cudaMemsetAsync(x->d_amax, 0, sizeof(unsigned) * xa.nsb * xa.nchan * xa.nsig, x->stream));
            FXC_CK(launch_fstage(x->cfg.nchan, x->spec_mode, fa, x->stream));
        }
        {
            StageScope sc(x, 2, fp8 ? 2 : 1);
            if (fp8) {
                // the e4m3 cast of the chunk belongs to the X operand: counted with the X stage
                FXC_CK(launch_cast_fp8(x->d_spec, x->d_amax, x->rows, x->nsig, x->T, xa.ntk, xa.nsb * xa.nchan,
                                       x->d_spec8, x->d_inv, x->stream));
                XArgs x8 = xa;
                x8.spec = x->d_spec8;
                x8.inv_scale = x->d_inv;
                FXC_CK(launch_xtc8(x8, x->d_err, x->nsm, x->stream));
            } else {
                FXC_CK(!tc ? launch_xplain(xa, x->stream)
                           : x->xf32 ? launch_xtc32(xa, x->d_err, x->nsm, x->stream)
                                     : launch_xtc(xa, x->d_err, x->nsm, x->stream));
            }
        }
    }
    return FXC_OK;
}

extern "C" {

int fxc_process_device(fxc_ctx* x, const uint8_t* d_data, size_t pitch, const double* delays,
                       const double* offs, int first, int nfft)
{
    if (!x || !d_data || pitch < x->subint + 16 || pitch % 16 || ((uintptr_t)d_data & 15)) return FXC_ERR_INVALID;
    FXC_CK(cudaSetDevice(x->device));
    return ctx_correlate(x, d_data, pitch, nullptr, delays, offs, first, nfft);
}

int fxc_process_device_window(fxc_ctx* x, const uint8_t* d_data, size_t pitch, const long long* base_sample,
                              size_t row_bytes, const double* delays, const double* offs, int first, int nfft)
{
    if (!x || !d_data || !base_sample || row_bytes == 0 || pitch < row_bytes + 32 || pitch % 16 ||
        ((uintptr_t)d_data & 15))
        return FXC_ERR_INVALID;
    const fxc_config& c = x->cfg;
    std::vector<long long> len(c.nant, (long long)row_bytes * 8 / sample_bits(c));
    for (int a = 0; a < c.nant; a++)
        if (base_sample[a] < 0 || base_sample[a] % sample_align(c)) return FXC_ERR_INVALID;
    FXC_CK(cudaSetDevice(x->device));
    // the caller's rows: the descriptor slot after the host windows', uploaded on the compute stream
    double* d_meta = x->d_win_meta + (size_t)fxc_ctx::NWIN * 2 * c.nant;
    const int st = upload_window_meta(x, base_sample, len.data(), d_meta, x->stream);
    if (st != FXC_OK) return st;
    return ctx_correlate(x, d_data, pitch, d_meta, delays, offs, first, nfft);
}

}  // extern "C"

// Sample range [lo, hi) antenna `a` needs for FFTs k0..k1 (kernel.c:373-386, 733-751 in
// plain double arithmetic).  The offset k*F - n(k) is quadratic in k (n follows the mean
// delay q k^2 + (q + l) k + ...), so its extremes lie at the ends of the range or around
// its vertex (F Ts - q - l) / 2q; widened by two samples for the +-1 offset nudges and
// rounding, and at the end by the unpacker's read-ahead byte.
static void window_range(const fxc_config& c, int F, const double* delays, const double* offs, int a, int k0,
                         int k1, long long& lo, long long& hi)
{
    const double q = delays[3 * a], l = delays[3 * a + 1], cc = delays[3 * a + 2];
    const double Ts = c.iscomplex ? 1.0 / c.bw : 1.0 / (2.0 * c.bw);
    auto offset = [&](double k) {
        const double mean = q * k * k + (q + l) * k + q / 2 + l / 2 + cc - q / 12;   // a/2 + b of kernel.c:383-385
        const double nf = (mean - offs[a]) / Ts;
        return (long long)k * F - (long long)std::trunc(nf + 0.5);
    };
    long long mn = std::min(offset(k0), offset(k1)), mx = std::max(offset(k0), offset(k1));
    if (q != 0.0) {
        const double kv = (F * Ts - q - l) / (2 * q);
        for (double k : {std::floor(kv), std::ceil(kv)})
            if (k > k0 && k < k1) {
                mn = std::min(mn, offset(k));
                mx = std::max(mx, offset(k));
            }
    }
    lo = mn - 2;
    hi = mx + F + 2 + tail_samples(c) + sample_align(c);
}

static int ensure_windows(fxc_ctx* x)
{
    if (x->d_win[0]) return FXC_OK;
    const fxc_config& c = x->cfg;
    // a window holds win_ffts FFTs plus the spread of their delays (far below an FFT for
    // sidereal rates) and the nudge margin: (win_ffts + 4) FFT lengths
    x->win_cap = (long long)(x->win_ffts + 4) * x->F;
    x->win_pitch = round_up((size_t)samples_to_bytes(c, x->win_cap) + 32, 256);
    const size_t bytes = (size_t)c.nsubband * c.nant * x->win_pitch;
    for (int s = 0; s < fxc_ctx::NWIN; s++) {
        FXC_CK(cudaMalloc(&x->d_win[s], bytes));
        FXC_CK(cudaEventCreateWithFlags(&x->win_ready[s], cudaEventDisableTiming));
        FXC_CK(cudaEventCreateWithFlags(&x->win_free[s], cudaEventDisableTiming));
    }
    FXC_CK(cudaStreamCreateWithFlags(&x->copy_stream, cudaStreamNonBlocking));
    return FXC_OK;
}

extern "C" {

int fxc_process_host_window(fxc_ctx* x, const uint8_t* const* data, const double* delays, const double* offs,
                            int first, int nfft)
{
    if (!x || !data || !delays || !offs || first < 0 || nfft < 1 || (long long)first + nfft > x->cfg.numffts)
        return FXC_ERR_INVALID;
    const fxc_config& c = x->cfg;
    for (int r = 0; r < c.nsubband * c.nant; r++)
        if (!data[r]) return FXC_ERR_INVALID;
    FXC_CK(cudaSetDevice(x->device));
    int st = ensure_windows(x);
    if (st != FXC_OK) return st;
    const int sal = sample_align(c);
    const long long total = (long long)x->subint * 8 / sample_bits(c);   // samples in a host row
    const int nrow = c.nsubband * c.nant;
    // rows evenly spaced in one host array: one strided copy per window over the union
    // of the antennas' ranges (when it fits), instead of one copy per row
    const ptrdiff_t rstride = nrow > 1 ? data[1] - data[0] : (ptrdiff_t)x->subint;
    bool uniform = rstride >= (ptrdiff_t)x->subint;
    for (int r = 1; r < nrow && uniform; r++) uniform = data[r] == data[0] + (ptrdiff_t)r * rstride;
    std::vector<long long> base(c.nant), len(c.nant);
    int k = first;
    int piece = x->win_ffts;
    while (k < first + nfft) {
        const int n = std::min(piece, first + nfft - k);
        bool fits = true;
        long long ulo = total, uhi = 0;
        for (int a = 0; a < c.nant && fits; a++) {
            long long lo, hi;
            window_range(c, x->F, delays, offs, a, k, k + n - 1, lo, hi);
            lo = std::max(0LL, std::min(lo, total));
            lo -= lo % sal;
            hi = std::max(lo, std::min(hi, total));
            base[a] = lo;
            len[a] = (hi - lo + sal - 1) / sal * sal;
            fits = len[a] <= x->win_cap;
            ulo = std::min(ulo, lo);
            uhi = std::max(uhi, base[a] + len[a]);
        }
        if (!fits) {   // delays that drift by more than the window margin: smaller pieces
            piece = std::max(1, n / 2);
            continue;
        }
        const int s = x->win_next;
        x->win_next = (s + 1) % fxc_ctx::NWIN;
        // copy stream: wait until the previous user of this window is done, then fill it and its
        // descriptor.  The descriptor goes on the copy stream too: an upload on the compute
        // stream would queue on the copy engine behind the window copies running ahead of it.
        FXC_CK(cudaStreamWaitEvent(x->copy_stream, x->win_free[s], 0));
        double* d_meta = x->d_win_meta + (size_t)s * 2 * c.nant;
        bool one_copy = false;
        if (uniform && uhi - ulo <= x->win_cap) {
            // rows that are equally spaced but separately allocated are refused by the strided
            // copy (its source range spans the allocations): per-row copies from then on
            one_copy = cudaMemcpy2DAsync(x->d_win[s], x->win_pitch, data[0] + samples_to_bytes(c, ulo),
                                         (size_t)rstride, (size_t)samples_to_bytes(c, uhi - ulo), nrow,
                                         cudaMemcpyHostToDevice,
                                         x->copy_stream) == cudaSuccess;
            if (!one_copy) {
                (void)cudaGetLastError();
                uniform = false;
            }
        }
        if (one_copy) {
            for (int a = 0; a < c.nant; a++) {
                base[a] = ulo;
                len[a] = uhi - ulo;
            }
        } else {
            for (int sb = 0; sb < c.nsubband; sb++)
                for (int a = 0; a < c.nant; a++) {
                    const int r = sb * c.nant + a;
                    FXC_CK(cudaMemcpyAsync(x->d_win[s] + (size_t)r * x->win_pitch,
                                           data[r] + samples_to_bytes(c, base[a]),
                                           (size_t)samples_to_bytes(c, len[a]), cudaMemcpyHostToDevice,
                                           x->copy_stream));
                }
        }
        st = upload_window_meta(x, base.data(), len.data(), d_meta, x->copy_stream);
        if (st != FXC_OK) return st;
        FXC_CK(cudaEventRecord(x->win_ready[s], x->copy_stream));
        FXC_CK(cudaStreamWaitEvent(x->stream, x->win_ready[s], 0));
        st = ctx_correlate(x, x->d_win[s], x->win_pitch, d_meta, delays, offs, k, n);
        if (st != FXC_OK) return st;
        FXC_CK(cudaEventRecord(x->win_free[s], x->stream));
        k += n;
    }
    return FXC_OK;
}

int fxc_upload_input(fxc_ctx* x, const uint8_t* const* data)
{
    if (!x || !data) return FXC_ERR_INVALID;
    if (!x->d_in) return FXC_ERR_UNSUPPORTED;
    FXC_CK(cudaSetDevice(x->device));
    const fxc_config& c = x->cfg;
    for (int r = 0; r < c.nsubband * c.nant; r++)
        if (!data[r]) return FXC_ERR_INVALID;
    for (int r = 0; r < c.nsubband * c.nant; r++)
        FXC_CK(cudaMemcpyAsync(x->d_in + (size_t)r * x->pitch, data[r], x->subint, cudaMemcpyHostToDevice,
                               x->stream));
    return FXC_OK;
}

int fxc_process_host(fxc_ctx* x, const uint8_t* const* data, const double* delays, const double* offs, int first,
                     int nfft)
{
    return fxc_process_host_window(x, data, delays, offs, first, nfft);
}

static void counts_out(fxc_ctx* x, const std::vector<int>& pc, int* counts)
{
    const int A = x->cfg.nant;
    int b = 0;
    auto pidx = [A](int a1, int a2) { return a1 * A - (a1 * (a1 - 1)) / 2 + (a2 - a1); };
    for (int a1 = 0; a1 < A - 1; a1++)
        for (int a2 = a1 + 1; a2 < A; a2++) counts[b++] = pc[pidx(a1, a2)];
    for (int a = 0; a < A; a++) counts[b++] = pc[pidx(a, a)];
}

}  // extern "C"

// Output of subbands [sb0, sb0 + nsb) into d_vis (layout of fxc_get_visibilities).
static int finalize_subbands(fxc_ctx* x, int sb0, int nsb, float* d_vis, int normalize)
{
    const fxc_config& c = x->cfg;
    StageScope sc(x, 3, 1);
    FXC_CK(launch_finalize(x->d_acc + (size_t)sb0 * x->npair * c.nchan, c.xmode != FXC_X_PLAIN_FP32 ? 1 : 0, x->nsig,
                           c.npol, c.nant, c.nchan, nsb, x->d_counts, normalize, reinterpret_cast<float2*>(d_vis),
                           x->stream));
    return FXC_OK;
}

extern "C" {

int fxc_get_visibilities_device(fxc_ctx* x, float* d_vis, int normalize)
{
    if (!x || !d_vis) return FXC_ERR_INVALID;
    FXC_CK(cudaSetDevice(x->device));
    return finalize_subbands(x, 0, x->cfg.nsubband, d_vis, normalize);
}

int fxc_get_visibilities(fxc_ctx* x, float* vis, int* counts, int normalize)
{
    if (!x || (!vis && !counts)) return FXC_ERR_INVALID;
    FXC_CK(cudaSetDevice(x->device));
    // one subband at a time through a one-subband device buffer (vis null: counts only)
    for (int sb = 0; vis && sb < x->cfg.nsubband; sb++) {
        const int st = finalize_subbands(x, sb, 1, reinterpret_cast<float*>(x->d_vis), normalize);
        if (st != FXC_OK) return st;
        FXC_CK(cudaMemcpyAsync(reinterpret_cast<char*>(vis) + (size_t)sb * x->vis_bytes, x->d_vis, x->vis_bytes,
                               cudaMemcpyDeviceToHost, x->stream));
    }
    std::vector<int> pc(x->npair_ant);
    FXC_CK(cudaMemcpyAsync(pc.data(), x->d_counts, sizeof(int) * x->npair_ant, cudaMemcpyDeviceToHost, x->stream));
    FXC_CK(cudaStreamSynchronize(x->stream));
    if (counts) counts_out(x, pc, counts);
    return device_status(x);
}

int fxc_get_amp_phase(fxc_ctx* x, float* ampphase, int normalize)
{
    if (!x || !ampphase) return FXC_ERR_INVALID;
    FXC_CK(cudaSetDevice(x->device));
    for (int sb = 0; sb < x->cfg.nsubband; sb++) {
        const int st = finalize_subbands(x, sb, 1, reinterpret_cast<float*>(x->d_vis), normalize);
        if (st != FXC_OK) return st;
        FXC_CK(launch_amp_phase(reinterpret_cast<float2*>(x->d_vis), (long long)(x->vis_bytes / sizeof(float2)),
                                x->stream));
        FXC_CK(cudaMemcpyAsync(reinterpret_cast<char*>(ampphase) + (size_t)sb * x->vis_bytes, x->d_vis, x->vis_bytes,
                               cudaMemcpyDeviceToHost, x->stream));
    }
    FXC_CK(cudaStreamSynchronize(x->stream));
    return device_status(x);
}

int fxc_set_plan(fxc_ctx* x, int fft_block, int x_variant)
{
    if (!x || (fft_block != 8 && fft_block != 16 && fft_block != 32) || (x_variant != 0 && x_variant != 1))
        return FXC_ERR_INVALID;
    x->plan_tb = fft_block;
    x->plan_alt = x_variant;
    return FXC_OK;
}

int fxc_get_plan(fxc_ctx* x, int* fft_block, int* x_variant)
{
    if (!x) return FXC_ERR_INVALID;
    if (fft_block) *fft_block = x->plan_tb;
    if (x_variant) *x_variant = x->plan_alt;
    return FXC_OK;
}

int fxc_autotune(fxc_ctx* x, int reps)
{
    if (!x || reps < 1) return FXC_ERR_INVALID;
    if (!x->model_valid) return FXC_ERR_INVALID;   // needs the input and delay model of an earlier call
    if (!x->d_in) return FXC_ERR_UNSUPPORTED;      // times on the whole-subintegration device input
    FXC_CK(cudaSetDevice(x->device));
    const fxc_config& c = x->cfg;
    const int nfft = std::min(x->T, c.numffts);
    int ld = 0;
    const std::vector<double> model = x->last_model;
    int st = ctx_run_delay_table(x, model.data(), model.data() + 3 * c.nant, 0, nfft, &ld);
    if (st != FXC_OK) return st;
    const bool tc = c.xmode != FXC_X_PLAIN_FP32;
    FArgs fa = ctx_fargs(x, x->d_in, x->pitch, ld);
    fa.t_base = 0;
    fa.nfft = nfft;
    fa.amax = x->d_amax;
    fa.nsb = x->nsb_g;   // the first subband group: what one chunk's spectra buffer holds
    cudaEvent_t e0, e1;
    FXC_CK(cudaEventCreate(&e0));
    FXC_CK(cudaEventCreate(&e1));
    auto timeit = [&](auto&& launch, float* ms) -> cudaError_t {
        cudaError_t e = launch();   // warm-up (also sets the kernel's shared-memory limit)
        if (e != cudaSuccess) return e;
        if ((e = cudaEventRecord(e0, x->stream)) != cudaSuccess) return e;
        for (int i = 0; i < reps; i++)
            if ((e = launch()) != cudaSuccess) return e;
        if ((e = cudaEventRecord(e1, x->stream)) != cudaSuccess) return e;
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) return e;
        return cudaEventElapsedTime(ms, e0, e1);
    };
    cudaError_t err = cudaSuccess;
    float best = 1e30f;
    int best_tb = x->plan_tb;
    for (int tb : {8, 16, 32}) {
        fa.tb = tb;
        float ms = 0.f;
        err = timeit([&] { return launch_fstage(c.nchan, x->spec_mode, fa, x->stream); }, &ms);
        if (err != cudaSuccess) break;
        if (ms < best) {
            best = ms;
            best_tb = tb;
        }
    }
    int best_alt = x->plan_alt;
    if (err == cudaSuccess && !tc) {
        XArgs xa{};
        xa.spec = x->d_spec;
        xa.acc = x->d_acc;
        xa.nsig = x->nsig;
        xa.T = x->T;
        xa.nchan = c.nchan;
        xa.nsb = x->nsb_g;
        xa.rows = x->rows;
        best = 1e30f;
        for (int alt : {0, 1}) {
            xa.alt = alt;
            ctx_xsegments(x, xa);
            float ms = 0.f;
            err = timeit([&] { return launch_xplain(xa, x->stream); }, &ms);
            if (err != cudaSuccess) break;
            if (ms < best) {
                best = ms;
                best_alt = alt;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess) {
        g_last_cuda = (int)err;
        return FXC_ERR_CUDA;
    }
    x->plan_tb = best_tb;
    x->plan_alt = best_alt;
    plan_cache_append({fplan_key(c) + " " + std::to_string(best_tb), xplan_key(x->nsig) + " " + std::to_string(best_alt)});
    return fxc_reset(x);   // the timing launches accumulated into the visibilities
}

int fxc_enable_stage_timing(fxc_ctx* x, int enable)
{
    if (!x) return FXC_ERR_INVALID;
    x->timing = enable != 0;
    return FXC_OK;
}

int fxc_stage_times(fxc_ctx* x, double* ms, long long* launches, int reset)
{
    if (!x) return FXC_ERR_INVALID;
    FXC_CK(cudaSetDevice(x->device));
    FXC_CK(cudaStreamSynchronize(x->stream));
    for (auto& p : x->pending) {
        float t = 0.f;
        FXC_CK(cudaEventElapsedTime(&t, p.a, p.b));
        x->stage_ms[p.stage] += t;
        x->event_pool.push_back(p.a);
        x->event_pool.push_back(p.b);
    }
    x->pending.clear();
    for (int s = 0; s < FXC_NSTAGE; s++) {
        if (ms) ms[s] = x->stage_ms[s];
        if (launches) launches[s] = x->stage_launches[s];
        if (reset) {
            x->stage_ms[s] = 0;
            x->stage_launches[s] = 0;
        }
    }
    return FXC_OK;
}

int fxc_debug_delay_table(fxc_ctx* x, const double* delays, const double* offs, int first, int nfft, int* offsets,
                          int* valid, double* frac, double* a, double* b)
{
    if (!x) return FXC_ERR_INVALID;
    FXC_CK(cudaSetDevice(x->device));
    int ld = 0;
    int st = ctx_run_delay_table(x, delays, offs, first, nfft, &ld);
    if (st != FXC_OK) return st;
    const int A = x->cfg.nant;
    std::vector<DelayEntry> h((size_t)A * ld);
    FXC_CK(cudaMemcpyAsync(h.data(), x->d_dtab, sizeof(DelayEntry) * h.size(), cudaMemcpyDeviceToHost, x->stream));
    FXC_CK(cudaStreamSynchronize(x->stream));
    for (int an = 0; an < A; an++)
        for (int t = 0; t < nfft; t++) {
            const DelayEntry& e = h[(size_t)an * ld + t];
            const size_t o = (size_t)an * nfft + t;
            if (offsets) offsets[o] = e.offset;
            if (valid) valid[o] = e.valid;
            if (frac) frac[o] = e.frac;
            if (a) a[o] = e.a;
            if (b) b[o] = e.b;
        }
    return FXC_OK;
}

int fxc_debug_unpack(fxc_ctx* x, const double* delays, const double* offs, int first, int nfft, float* out)
{
    if (!x || !out) return FXC_ERR_INVALID;
    if (!x->d_in || x->cfg.iscomplex) return FXC_ERR_UNSUPPORTED;
    FXC_CK(cudaSetDevice(x->device));
    int ld = 0;
    int st = ctx_run_delay_table(x, delays, offs, first, nfft, &ld);
    if (st != FXC_OK) return st;
    const fxc_config& c = x->cfg;
    const size_t n = (size_t)c.nsubband * c.nant * c.npol * nfft * x->F;
    float* d = nullptr;
    FXC_CK(cudaMalloc(&d, n * sizeof(float)));
    FArgs fa = ctx_fargs(x, x->d_in, x->pitch, ld);
    fa.t_base = 0;
    fa.nfft = nfft;
    cudaError_t e = launch_unpack_debug(c.nchan, fa, d, x->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, n * sizeof(float), cudaMemcpyDeviceToHost, x->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(x->stream);
    cudaFree(d);
    FXC_CK(e);
    return FXC_OK;
}

int fxc_debug_expire_wait(fxc_ctx* x)
{
    if (!x) return FXC_ERR_INVALID;
    FXC_CK(cudaSetDevice(x->device));
    FXC_CK(launch_expire_wait(x->d_err, x->stream));
    return FXC_OK;
}

int fxc_debug_expire_wait_tc(fxc_ctx* x)
{
    if (!x) return FXC_ERR_INVALID;
    FXC_CK(cudaSetDevice(x->device));
    FXC_CK(launch_expire_wait_tc(x->d_err, x->stream));
    return FXC_OK;
}

int fxc_debug_spectra(fxc_ctx* x, const double* delays, const double* offs, int first, int nfft, float* out)
{
    if (!x || !out || nfft > x->T) return FXC_ERR_INVALID;
    if (!x->d_in) return FXC_ERR_UNSUPPORTED;
    FXC_CK(cudaSetDevice(x->device));
    int ld = 0;
    int st = ctx_run_delay_table(x, delays, offs, first, nfft, &ld);
    if (st != FXC_OK) return st;
    const fxc_config& c = x->cfg;
    const int T = (int)round_up((size_t)nfft, 64);
    const size_t n = (size_t)c.nsubband * x->nsig * T * c.nchan;
    float2* d = nullptr;
    FXC_CK(cudaMalloc(&d, n * sizeof(float2)));
    FArgs fa = ctx_fargs(x, x->d_in, x->pitch, ld);
    fa.t_base = 0;
    fa.nfft = nfft;
    fa.T = T;
    fa.spec = d;
    if (fa.fkind == FXC_F_TC16) fa.fkind = FXC_F_FFT32;   // the FP16 tensor-core DFT has no FP32 output
    cudaError_t e = launch_fstage(c.nchan, kSpecF32, fa, x->stream);
    for (int r = 0; e == cudaSuccess && r < c.nsubband * x->nsig; r++)
        e = cudaMemcpyAsync(out + (size_t)r * nfft * c.nchan * 2, d + (size_t)r * T * c.nchan,
                            sizeof(float2) * nfft * c.nchan, cudaMemcpyDeviceToHost, x->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(x->stream);
    cudaFree(d);
    FXC_CK(e);
    return FXC_OK;
}

}  // extern "C"
