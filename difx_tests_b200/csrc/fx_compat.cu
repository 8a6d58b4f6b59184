// fx_compat.cu -- the reference's kernel.h entry points over the C ABI
// (include/fxkernel_compat.h), so a host written for kernel.c (main.c) links
// against libfxcorr.so unchanged.  Host code only; every FX stage runs on the GPU
// through fxc_process_host.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>

#include "../../include/fxcorr.h"
#include "../../include/fxkernel_compat.h"

namespace {

int g_compat_status = FXC_OK;

// One cached context (the reference is single-threaded and processes one geometry).
struct CompatState {
    fxc_ctx* ctx = nullptr;
    fxc_config cfg{};
    std::vector<float> vis;
    std::vector<int> counts;
    std::vector<double> delays;
} g;

bool same_cfg(const fxc_config& a, const fxc_config& b)
{
    return a.nant == b.nant && a.npol == b.npol && a.nchan == b.nchan && a.numffts == b.numffts &&
           a.nsubband == b.nsubband && a.xmode == b.xmode && a.lo == b.lo && a.bw == b.bw;
}

int fail(const char* what, int st)
{
    std::fprintf(stderr, "fxcorr: %s: %s\n", what, fxc_strerror(st));
    g_compat_status = st;
    return st;
}

fxc_cf32** alloc_rows(int nrows, int n)
{
    fxc_cf32** p = (fxc_cf32**)std::malloc(sizeof(fxc_cf32*) * nrows);
    if (!p) return nullptr;
    for (int r = 0; r < nrows; r++) {
        p[r] = (fxc_cf32*)std::calloc((size_t)n, sizeof(fxc_cf32));
        if (!p[r]) return nullptr;
    }
    return p;
}

}  // namespace

extern "C" {

int fxc_compat_last_error(void) { return g_compat_status; }

void startTiming(struct timespec* starttime, char* starttimestring)
{
    // kernel.c:649-654
    clock_gettime(CLOCK_MONOTONIC, starttime);
    const time_t now = time(nullptr);
    std::strftime(starttimestring, 64, "%c", std::localtime(&now));
}

void endTiming(struct timespec* starttime, long long* diff_ms)
{
    // kernel.c:656-667: prints ms, then leaves microseconds in *diff_ms
    struct timespec end;
    clock_gettime(CLOCK_MONOTONIC, &end);
    const long long ns = (end.tv_sec - starttime->tv_sec) * 1000000000LL + (end.tv_nsec - starttime->tv_nsec);
    std::printf("Run time was %lld milliseconds\n", ns / 1000000LL);
    *diff_ms = ns / 1000LL;
    std::printf("Run time was %lld microsec\n", *diff_ms);
}

void saveLog(long long* diff_ms, char* starttimestring)
{
    // kernel.c:632-647
    FILE* f = std::fopen("runtime.fxkernel.log", "w");
    if (!f) {
        std::fprintf(stderr, "Error opening file for writing\n");
        return;
    }
    std::fprintf(f, "Run time was %lld milliseconds\n", *diff_ms);
    std::fprintf(f, "Start time was %s\n", starttimestring);
    std::fclose(f);
}

void resetBeforeProcess(int* nbaselines, fxc_cf32*** visibilities, int* nchan, int* baselineCount, int split)
{
    for (int i = 0; i < split * *nbaselines; i++)
        for (int j = 0; j < 4; j++) std::memset(visibilities[i][j], 0, sizeof(fxc_cf32) * (size_t)*nchan);
    std::memset(baselineCount, 0, sizeof(int) * (size_t)split * *nbaselines);
}

void init_FxKernel(int* nant, int* nchan, int* nbit, double* lo, double* bw, struct timespec* starttime,
                   char* starttimestring, int* fftchannels, double* sampletime, int* stridesize, int* substridesize,
                   int* fractionalLoFreq, fxc_cf32*** unpacked, fxc_cf32*** channelised, fxc_cf32*** conjchannels,
                   fxc_cf32*** visibilities, int* nbaselines, int* baselineCount, int split)
{
    g_compat_status = FXC_OK;
    // derived sizes, kernel.c:13-39
    *fftchannels = 2 * *nchan;
    *sampletime = 1.0 / (2.0 * *bw);
    if (*nbit != 2) {
        fail("init_FxKernel: only 2-bit data is supported", FXC_ERR_UNSUPPORTED);
        return;
    }
    if (*nchan < 128 || *nchan > 4096 || (*nchan & (*nchan - 1))) {
        fail("init_FxKernel: nchan must be a power of two in [128, 4096]", FXC_ERR_INVALID);
        return;
    }
    *stridesize = (int)std::sqrt((double)*nchan);
    *substridesize = 2 * *stridesize;
    *fractionalLoFreq = (*lo - (int)(*lo)) > 0.00000000001;
    // host arrays the reference host expects (kernel.c:41-110)
    for (int i = 0; i < split * *nant; i++) {
        unpacked[i] = alloc_rows(2, *fftchannels);
        channelised[i] = alloc_rows(2, *fftchannels);
        conjchannels[i] = alloc_rows(2, *nchan);
        if (!unpacked[i] || !channelised[i] || !conjchannels[i]) {
            fail("init_FxKernel: host allocation", FXC_ERR_NOMEM);
            return;
        }
    }
    *nbaselines = *nant * (*nant - 1) / 2;
    for (int i = 0; i < split * *nbaselines; i++) {
        visibilities[i] = alloc_rows(4, *nchan);
        if (!visibilities[i]) {
            fail("init_FxKernel: host allocation", FXC_ERR_NOMEM);
            return;
        }
    }
    startTiming(starttime, starttimestring);
    resetBeforeProcess(nbaselines, visibilities, nchan, baselineCount, split);
}

void processAntennasAndBaselinePara(int* nant, int* numffts, int* fftchannels, double* antFileOffsets,
                                    double* sampletime, unsigned char** inputData, fxc_cf32*** unpacked,
                                    fxc_cf32*** channelised, fxc_cf32*** conjchannels, double** delays, int* nbit,
                                    int* substridesize, int* stridesize, int* fractionalLoFreq, double* lo,
                                    int* nchan, fxc_cf32*** visibilities, int* baselineCount, int* iteration,
                                    double* bw, fxc_cf32*** visibilities_out, int* baselineCount_out, int split)
{
    (void)fftchannels; (void)sampletime; (void)unpacked; (void)channelised; (void)conjchannels;
    (void)substridesize; (void)stridesize; (void)fractionalLoFreq;
    const int A = *nant;
    const int nbl = A * (A - 1) / 2;
    fxc_config cfg;
    fxc_config_default(&cfg);
    cfg.nant = A;
    cfg.npol = 2;                       // the reference always reads interleaved dual-pol data (kernel.c:397-426)
    cfg.nchan = *nchan;
    cfg.nbit = *nbit;
    cfg.numffts = *numffts * split;     // the subintegration; sets maxoffset (kernel.c:730)
    cfg.lo = *lo;
    cfg.bw = *bw;
    cfg.sb_spacing = *bw;
    const char* xm = std::getenv("FXC_COMPAT_XMODE");
    cfg.xmode = !xm ? FXC_X_PLAIN_FP32
              : std::strcmp(xm, "tc") == 0 ? FXC_X_TC_FP16
              : std::strcmp(xm, "fp8") == 0 ? FXC_X_TC_FP8 : FXC_X_PLAIN_FP32;
    int st;
    if (!g.ctx || !same_cfg(g.cfg, cfg)) {
        if (g.ctx) fxc_destroy(g.ctx);
        g.ctx = nullptr;
        if ((st = fxc_create(&cfg, &g.ctx)) != FXC_OK) {
            fail("processAntennasAndBaselinePara: fxc_create", st);
            return;
        }
        g.cfg = cfg;
        g.vis.assign(2 * fxc_vis_count(&cfg), 0.f);
        g.counts.assign(nbl + A, 0);
    }
    g.delays.resize(3 * (size_t)A);
    for (int a = 0; a < A; a++)
        for (int k = 0; k < 3; k++) g.delays[3 * a + k] = delays[a][k];
    if ((st = fxc_reset(g.ctx)) != FXC_OK || (st = fxc_upload_input(g.ctx, inputData)) != FXC_OK) {
        fail("processAntennasAndBaselinePara: upload", st);
        return;
    }
    // iteration[] holds absolute FFT indices; process each contiguous run
    uint8_t* d_in = nullptr;
    size_t pitch = 0;
    fxc_device_input(g.ctx, &d_in, &pitch);
    for (int k0 = 0; k0 < *numffts;) {
        int k1 = k0 + 1;
        while (k1 < *numffts && iteration[k1] == iteration[k1 - 1] + 1) k1++;
        st = fxc_process_device(g.ctx, d_in, pitch, g.delays.data(), antFileOffsets, iteration[k0], k1 - k0);
        if (st != FXC_OK) {
            fail("processAntennasAndBaselinePara: fxc_process_device", st);
            return;
        }
        k0 = k1;
    }
    if ((st = fxc_get_visibilities(g.ctx, g.vis.data(), g.counts.data(), 0)) != FXC_OK) {
        fail("processAntennasAndBaselinePara: fxc_get_visibilities", st);
        return;
    }
    // accumulate like processBaselinePara (kernel.c:829-854): crosses only, product 2l+m
    const int C = *nchan;
    for (int b = 0; b < nbl; b++) {
        for (int p = 0; p < 4; p++) {
            const float* src = g.vis.data() + 2 * ((size_t)(b * 4 + p) * C);
            fxc_cf32* dst = visibilities[b][p];
            for (int c = 0; c < C; c++) {
                dst[c].re += src[2 * c];
                dst[c].im += src[2 * c + 1];
            }
        }
        baselineCount[b] += g.counts[b];
    }
    // shallow copies, as kernel.c:825-826
    std::memcpy(visibilities_out, visibilities, sizeof(fxc_cf32**) * nbl);
    std::memcpy(baselineCount_out, baselineCount, sizeof(int) * nbl);
}

void merge(int split, int nbaselines, fxc_cf32*** visibilities, int* nant, int* nChan, int* baselineCount,
           fxc_cf32*** visibilities_out, int* baselineCount_out)
{
    // kernel.c:856-878: sum the split partials into the first slice
    const int nbl = *nant * (*nant - 1) / 2;
    if (split != 1) {
        for (int i = 0; i < nbaselines; i++) {
            for (int j = 0; j < 4; j++)
                for (int k = 1; k < split; k++)
                    for (int c = 0; c < *nChan; c++) {
                        visibilities[i][j][c].re += visibilities[i + k * nbl][j][c].re;
                        visibilities[i][j][c].im += visibilities[i + k * nbl][j][c].im;
                    }
            for (int k = 1; k < split; k++) baselineCount[i] += baselineCount[i + k * nbaselines];
        }
    }
    std::memcpy(visibilities_out, visibilities, sizeof(fxc_cf32**) * nbl);
    std::memcpy(baselineCount_out, baselineCount, sizeof(int) * nbl);
}

void processNormalize(int* nbaselines, int* baselineCount, fxc_cf32*** visibilities, int* nchan,
                      fxc_cf32*** visibilities_out)
{
    // kernel.c:348-359: divide by the count, skip baselines without data
    for (int i = 0; i < *nbaselines; i++) {
        if (baselineCount[i] == 0) continue;
        const float n = (float)baselineCount[i];
        for (int j = 0; j < 4; j++)
            for (int c = 0; c < *nchan; c++) {
                visibilities[i][j][c].re /= n;
                visibilities[i][j][c].im /= n;
            }
    }
    std::memcpy(visibilities_out, visibilities, sizeof(fxc_cf32**) * (size_t)*nbaselines);
}

void saveVisibilities(int* nbaselines, int* nchan, fxc_cf32*** visibilities, double* bw)
{
    // kernel.c:570-630: per channel "%5d %11.6f" then per baseline x product re, im, amp, phase
    FILE* f = std::fopen("vis.out", "w");
    if (!f) {
        std::fprintf(stderr, "Error opening file for writing.\n");
        return;
    }
    for (int c = 0; c < *nchan; c++) {
        std::fprintf(f, "%5d %11.6f", c, (c + 0.5) / *nchan * *bw / 1e6);
        for (int i = 0; i < *nbaselines; i++)
            for (int j = 0; j < 4; j++) {
                const fxc_cf32 v = visibilities[i][j][c];
                const float amp = std::sqrt(v.re * v.re + v.im * v.im);
                const float ph = std::atan2(v.im, v.re);
                std::fprintf(f, " %11.6f %11.6f", v.re, v.im);
                std::fprintf(f, " %11.6f %10.6f", amp, ph);
            }
        std::fprintf(f, "\n");
    }
    std::fclose(f);
}

}  // extern "C"
