// fx_noalloc.cu -- one-shot correlation that allocates no device memory.
//
// Some callers cannot allocate GPU memory at the point they want to correlate:
// real-time paths that must not take the allocator's locks or wait on its
// latency, and hosts whose device memory another framework reserved up front
// (an allocation there fails or evicts that framework's pool).
// fxc_correlate_noalloc serves them: the caller passes the packed input and the
// output buffers (device memory it already owns); every intermediate (delay
// model, delay table, validity bits, baseline counts, accumulators, spectra, and
// an error word) lives in one file-scope __device__ array of
// FXC_NOALLOC_SCRATCH_BYTES.
//
// The array is part of the library image, so every GPU that loads this library
// holds it until the process exits.  All calls share it and it keeps the last
// call's contents: every region that must start at zero is cleared at the start
// of each call, and two calls that overlap on the GPU (different streams, or
// different host threads without ordering) race on it.
//
// In host code the array's name is only a host-side stand-in; its device
// address is obtained once per device with cudaGetSymbolAddress (with that
// device current) and cached by the first call on that device.
//
// A bounded device wait of the F stage that runs out (its input copy never
// completed) is reported in the outputs, since the call returns before the GPU
// finishes: every visibility becomes NaN and every entry of d_counts (when
// given) becomes -6.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/fxcorr.h"
#include "fx_internal.h"
#include "fx_kernels.h"

using namespace fx;

static __device__ __align__(256) unsigned char g_fx_noalloc_scratch[FXC_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
unsigned char* g_scratch_dev[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of the scratch array on the current device (looked up once).
cudaError_t scratch_address(int dev, unsigned char** out)
{
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_dev[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_fx_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_dev[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_dev[dev];
    return cudaSuccess;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// counts per antenna pair (row-major upper triangle incl. autos) -> output
// baseline order: crosses as the reference orders them (kernel.c:832-852), then autos
__global__ void k_counts_to_output(const int* __restrict__ pair_counts, int nant, int* __restrict__ out)
{
    const int nbl = nant * (nant - 1) / 2;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbl + nant; b += gridDim.x * blockDim.x) {
        int a1, a2;
        if (b < nbl) {
            int rem = b;
            a1 = 0;
            while (rem >= nant - 1 - a1) {
                rem -= nant - 1 - a1;
                a1++;
            }
            a2 = a1 + 1 + rem;
        } else {
            a1 = a2 = b - nbl;
        }
        out[b] = pair_counts[a1 * nant - (a1 * (a1 - 1)) / 2 + (a2 - a1)];
    }
}

// An expired device wait (error word != 0) poisons the outputs: NaN visibilities and
// counts of -code, so a caller that cannot synchronise on the call still sees it.
__global__ void k_noalloc_flag_error(const int* __restrict__ err, float* __restrict__ vis, size_t nvis_floats,
                                     int* __restrict__ counts, int ncounts)
{
    const int code = *err;
    if (code == 0) return;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t nth = (size_t)gridDim.x * blockDim.x;
    for (size_t i = tid; i < nvis_floats; i += nth) vis[i] = __int_as_float(0x7fc00000);
    if (counts)
        for (size_t i = tid; i < (size_t)ncounts; i += nth) counts[i] = -code;
}

}  // namespace

#define NA_CK(call)                                   \
    do {                                              \
        const cudaError_t e_ = (call);                \
        if (e_ != cudaSuccess) return FXC_ERR_CUDA;   \
    } while (0)

extern "C" int fxc_correlate_noalloc(const fxc_config* cfg, const uint8_t* d_data, size_t pitch, const double* delays,
                                     const double* fileoffsets, int first_fft, int nfft, float* d_vis, int* d_counts,
                                     int normalize, void* stream)
{
    if (!cfg || !d_data || !delays || !fileoffsets || !d_vis) return FXC_ERR_INVALID;
    const fxc_config& c = *cfg;
    if (c.nant < 2 || c.npol < 1 || c.npol > 2 || c.numffts < 1 || c.nsubband < 1) return FXC_ERR_INVALID;
    if (c.nchan < 128 || c.nchan > 4096 || (c.nchan & (c.nchan - 1))) return FXC_ERR_INVALID;
    if (c.nbit != 2 || c.iscomplex != 0 || c.xmode != FXC_X_PLAIN_FP32) return FXC_ERR_UNSUPPORTED;
    if (c.nant * c.npol > 64) return FXC_ERR_UNSUPPORTED;
    if (!(c.bw > 0.0) || !std::isfinite(c.lo) || !std::isfinite(c.sb_spacing)) return FXC_ERR_INVALID;
    if ((long long)(c.numffts + 1) * 2 * c.nchan > 0x7fffffffLL) return FXC_ERR_INVALID;
    if (first_fft < 0 || nfft < 1 || (long long)first_fft + nfft > c.numffts) return FXC_ERR_INVALID;
    for (int i = 0; i < 3 * c.nant; i++)
        if (!std::isfinite(delays[i])) return FXC_ERR_INVALID;
    for (int i = 0; i < c.nant; i++)
        if (!std::isfinite(fileoffsets[i])) return FXC_ERR_INVALID;
    const size_t subint = fxc_subint_bytes(cfg);
    if (pitch < subint + 16 || pitch % 16 || ((uintptr_t)d_data & 15)) return FXC_ERR_INVALID;

    // ---- scratch layout (offsets 256-byte aligned)
    const int F = 2 * c.nchan;
    const int nsig = c.nant * c.npol;
    const int npair = nsig * (nsig + 1) / 2;
    const int npair_ant = c.nant * (c.nant + 1) / 2;
    const int ld = (int)(((size_t)nfft + 127) / 128 * 128);
    const int stride = 1 << ((int)std::log2((double)c.nchan) / 2);
    size_t off = 0;
    const size_t o_err = off;     off = align256(off + sizeof(int));
    const size_t o_model = off;   off = align256(off + 4 * sizeof(double) * c.nant);
    const size_t o_sblo = off;    off = align256(off + sizeof(double) * c.nsubband);
    const size_t o_csub = off;    off = align256(off + sizeof(float) * stride);
    const size_t o_cstep = off;   off = align256(off + sizeof(float) * (c.nchan / stride));
    const size_t o_dtab = off;    off = align256(off + sizeof(DelayEntry) * (size_t)c.nant * ld);
    const size_t o_vbits = off;   off = align256(off + sizeof(uint32_t) * (size_t)c.nant * (ld / 32));
    const size_t o_counts = off;  off = align256(off + sizeof(int) * npair_ant);
    const size_t o_acc = off;     off = align256(off + sizeof(float2) * (size_t)c.nsubband * npair * c.nchan);
    const size_t o_spec = off;
    const size_t per_slot = sizeof(float2) * (size_t)c.nsubband * nsig * c.nchan;
    if (o_spec >= FXC_NOALLOC_SCRATCH_BYTES) return FXC_ERR_INVALID;   // problem too large for the scratch
    size_t T = (FXC_NOALLOC_SCRATCH_BYTES - o_spec) / per_slot / 64 * 64;
    if (T < 64) return FXC_ERR_INVALID;                                   // problem too large for the scratch
    T = std::min(T, ((size_t)nfft + 63) / 64 * 64);

    int dev = 0;
    NA_CK(cudaGetDevice(&dev));
    unsigned char* scratch = nullptr;
    NA_CK(scratch_address(dev, &scratch));
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // ---- constants and delay model into scratch; zero what accumulates
    std::vector<double> model(4 * (size_t)c.nant), sblo(c.nsubband);
    std::memcpy(model.data(), delays, 3 * sizeof(double) * c.nant);
    std::memcpy(model.data() + 3 * c.nant, fileoffsets, sizeof(double) * c.nant);
    for (int s = 0; s < c.nsubband; s++) sblo[s] = c.lo + c.sb_spacing * s;
    std::vector<float> csub(stride), cstep(c.nchan / stride);
    const double two_pi = 2 * 3.14159265358979323846;
    for (int j = 0; j < stride; j++) csub[j] = (float)((two_pi * j * c.bw) / (double)c.nchan);
    for (int i = 0; i < c.nchan / stride; i++) cstep[i] = (float)((two_pi * i * stride * c.bw) / (double)c.nchan);
    NA_CK(cudaMemcpyAsync(scratch + o_model, model.data(), model.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(scratch + o_sblo, sblo.data(), sblo.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(scratch + o_csub, csub.data(), csub.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(scratch + o_cstep, cstep.data(), cstep.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemsetAsync(scratch + o_err, 0, sizeof(int), st));
    NA_CK(cudaMemsetAsync(scratch + o_counts, 0, sizeof(int) * npair_ant, st));
    NA_CK(cudaMemsetAsync(scratch + o_acc, 0, sizeof(float2) * (size_t)c.nsubband * npair * c.nchan, st));
    NA_CK(cudaMemsetAsync(scratch + o_spec, 0, per_slot * T, st));

    // ---- the same stages as fxc_process_device + fxc_get_visibilities_device
    const double* d_model = reinterpret_cast<const double*>(scratch + o_model);
    DelayEntry* d_dtab = reinterpret_cast<DelayEntry*>(scratch + o_dtab);
    uint32_t* d_vbits = reinterpret_cast<uint32_t*>(scratch + o_vbits);
    int* d_pc = reinterpret_cast<int*>(scratch + o_counts);
    float2* d_acc = reinterpret_cast<float2*>(scratch + o_acc);
    NA_CK(launch_delay_table(d_model, d_model + 3 * c.nant, nullptr, first_fft, c.nant, nfft, ld, F,
                             (c.numffts - 1) * F, 1.0 / (2.0 * c.bw), d_dtab, d_vbits, st));
    NA_CK(launch_counts(d_vbits, c.nant, ld / 32, d_pc, st));
    FArgs fa;
    std::memset(&fa, 0, sizeof(fa));
    fa.data = d_data;
    fa.pitch = pitch;
    fa.dtab = d_dtab;
    fa.ld = ld;
    fa.nant = c.nant;
    fa.npol = c.npol;
    fa.nsb = c.nsubband;
    fa.sb_lo = reinterpret_cast<const double*>(scratch + o_sblo);
    fa.chan_sub = reinterpret_cast<const float*>(scratch + o_csub);
    fa.chan_step = reinterpret_cast<const float*>(scratch + o_cstep);
    fa.spec = scratch + o_spec;
    fa.T = (int)T;
    fa.err = reinterpret_cast<int*>(scratch + o_err);
    XArgs xa{};
    xa.spec = scratch + o_spec;
    xa.acc = d_acc;
    xa.nsig = nsig;
    xa.T = (int)T;
    xa.nchan = c.nchan;
    xa.nsb = c.nsubband;
    xa.rows = 0;
    for (int c0 = 0; c0 < nfft; c0 += (int)T) {
        fa.t_base = c0;
        fa.nfft = std::min((int)T, nfft - c0);
        NA_CK(launch_fstage(c.nchan, kSpecF32, fa, st));
        NA_CK(launch_xplain(xa, st));
    }
    NA_CK(launch_finalize(d_acc, 0, nsig, c.npol, c.nant, c.nchan, c.nsubband, d_pc, normalize,
                          reinterpret_cast<float2*>(d_vis), st));
    const int nout = c.nant * (c.nant - 1) / 2 + c.nant;
    if (d_counts) {
        k_counts_to_output<<<(nout + 255) / 256, 256, 0, st>>>(d_pc, c.nant, d_counts);
        NA_CK(cudaGetLastError());
    }
    k_noalloc_flag_error<<<148, 256, 0, st>>>(reinterpret_cast<const int*>(scratch + o_err), d_vis,
                                              2 * fxc_vis_count(cfg), d_counts, nout);
    NA_CK(cudaGetLastError());
    return FXC_OK;
}
