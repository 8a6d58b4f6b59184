// fx_delay.cu -- K0 (delay table), baseline counts and the finalise step.
#include "fx_common.cuh"
#include "fx_kernels.h"

namespace fx {

// K0: one thread per (antenna, FFT).  Reproduces kernel.c:373-386 (station
// delay: quadratic evaluated at FFT start/middle/end -> linear model a, b and
// mean) and kernel.c:733-756 (integer offset with C truncation, fractional
// delay, the offset == -1 / maxoffset+1 nudges, validity) in IEEE binary64
// with every operation rounded separately, as gcc compiles it on x86-64.
//
// Input windows: the rows of antenna `ant` start at subintegration sample
// win[ant] and hold win[nant + ant] samples (win null: the whole subintegration
// from sample 0); the table stores offsets relative to the window.  A reference-valid FFT whose samples (plus the one-byte
// read-ahead of kernel.c:402-409) are not all in the window is marked invalid
// and raises bit kWindowMiss in *err, so nothing outside the rows is read.
__global__ void k_delay_table(const double* __restrict__ delays, const double* __restrict__ fileoffsets,
                              const int* __restrict__ fftindex, int first, int nfft, int ld, int F, int maxoffset,
                              double sampletime, const double* __restrict__ win, int nant, int spb,
                              int* __restrict__ err, DelayEntry* __restrict__ tab, uint32_t* __restrict__ vbits)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int ant = blockIdx.y;
    int valid = 0;
    if (t < nfft) {
        const double q = delays[3 * ant + 0], l = delays[3 * ant + 1], c = delays[3 * ant + 2];
        const int k = fftindex ? fftindex[t] : first + t;
        const double kd = (double)k;
        const double d0 = dadd(dadd(dmul(dmul(q, kd), kd), dmul(l, kd)), c);
        const double kh = dadd(kd, 0.5);
        const double d1 = dadd(dadd(dmul(dmul(q, kh), kh), dmul(l, kh)), c);
        const double k1 = dadd(kd, 1.0);
        const double d2 = dadd(dadd(dmul(dmul(q, k1), k1), dmul(l, k1)), c);
        const double a = dsub(d2, d0);
        const double b = dadd(d0, ddiv(dsub(d1, dadd(dmul(a, 0.5), d0)), 3.0));
        const double mean = dadd(dmul(a, 0.5), b);
        const double nf = ddiv(dsub(mean, fileoffsets[ant]), sampletime);
        const int n = dtrunc_int(dadd(nf, 0.5));
        double frac = dmul(-dsub(nf, (double)n), sampletime);
        int offset = k * F - n;
        if (offset == -1) {
            offset = 0;
            frac = dadd(frac, sampletime);
        }
        if (offset == maxoffset + 1) {
            offset = offset - 1;
            frac = dsub(frac, sampletime);
        }
        valid = (offset >= 0 && offset <= maxoffset) ? 1 : 0;
        if (win) {
            const long long rel = (long long)offset - (long long)win[ant];
            if (valid && (rel < 0 || rel + F + spb > (long long)win[nant + ant])) {
                valid = 0;
                atomicOr(err, kWindowMiss);
            }
            offset = (int)rel;
        }
        DelayEntry e;
        e.a = a;
        e.b = b;
        e.frac = frac;
        e.offset = offset;
        e.valid = valid;
        tab[(size_t)ant * ld + t] = e;
    }
    const uint32_t m = __ballot_sync(0xffffffffu, valid != 0);
    if ((threadIdx.x & 31) == 0 && t < ld) vbits[(size_t)ant * (ld / 32) + (t >> 5)] = m;
}

// counts[pair(a1, a2)] += #FFTs with both antennas valid (kernel.c:850), a1 <= a2
__global__ void k_counts(const uint32_t* __restrict__ vbits, int nant, int nwords, int* __restrict__ counts)
{
    const int p = blockIdx.x;  // antenna pair, row-major upper triangle incl. diagonal
    int a1 = 0, rem = p;
    while (rem >= nant - a1) {
        rem -= nant - a1;
        a1++;
    }
    const int a2 = a1 + rem;
    int c = 0;
    for (int w = threadIdx.x; w < nwords; w += blockDim.x)
        c += __popc(vbits[(size_t)a1 * nwords + w] & vbits[(size_t)a2 * nwords + w]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ int part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += part[i];
        counts[p] += s;
    }
}

__device__ __forceinline__ int pair_index(int i, int j, int n)  // i <= j
{
    return i * n - (i * (i - 1)) / 2 + (j - i);
}

__device__ __forceinline__ int ant_pair_index(int a1, int a2, int nant) { return pair_index(a1, a2, nant); }

// Output: vis[sb][bl][prod][nchan] complex, bl = crosses in reference order
// (kernel.c:832-852) then autos; prod = 2*l + m (kernel.c:846).  Optional
// normalisation by the baseline count (kernel.c:348-359).
__global__ void k_finalize(const float2* __restrict__ acc, int acc_layout, int nsig, int npol, int nant,
                           int nchan, int nsb, const int* __restrict__ counts, int normalize,
                           float2* __restrict__ vis)
{
    const int nbl = nant * (nant - 1) / 2;
    const int nout = nbl + nant;
    const int np2 = npol * npol;
    const size_t total = (size_t)nsb * nout * np2 * nchan;
    const int npair = nsig * (nsig + 1) / 2;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % nchan);
        size_t r = e / nchan;
        const int prod = (int)(r % np2);
        r /= np2;
        const int bl = (int)(r % nout);
        const int sb = (int)(r / nout);
        int a1, a2;
        if (bl < nbl) {
            // row a1 of the strict upper triangle starts at S(a1) = a1 (2 nant - a1 - 1) / 2
            const double m = 2.0 * nant - 1.0;
            a1 = (int)((m - sqrt(m * m - 8.0 * bl)) * 0.5);
            if (a1 < 0) a1 = 0;
            while (a1 > 0 && a1 * (2 * nant - a1 - 1) / 2 > bl) a1--;
            while ((a1 + 1) * (2 * nant - a1 - 2) / 2 <= bl) a1++;
            a2 = a1 + 1 + (bl - a1 * (2 * nant - a1 - 1) / 2);
        } else {
            a1 = a2 = bl - nbl;
        }
        const int l = prod / npol, m = prod % npol;
        int i = a1 * npol + l, j = a2 * npol + m;
        bool conj = false;
        if (i > j) {
            const int tmp = i;
            i = j;
            j = tmp;
            conj = true;
        }
        const int p = pair_index(i, j, nsig);
        float2 v = (acc_layout == 0) ? acc[((size_t)sb * npair + p) * nchan + c]
                                     : acc[((size_t)sb * nchan + c) * npair + p];
        if (conj) v.y = -v.y;
        if (normalize) {
            const int cnt = counts[ant_pair_index(a1, a2, nant)];
            if (cnt != 0) {
                v.x = v.x / (float)cnt;
                v.y = v.y / (float)cnt;
            }
        }
        vis[e] = v;
    }
}

cudaError_t launch_delay_table(const double* delays, const double* fileoffsets, const int* fftindex, int first,
                               int nant, int nfft, int ld, int F, int maxoffset, double sampletime, DelayEntry* tab,
                               uint32_t* vbits, cudaStream_t st)
{
    return launch_delay_table_window(delays, fileoffsets, fftindex, first, nant, nfft, ld, F, maxoffset, sampletime,
                                     nullptr, 0, nullptr, tab, vbits, st);
}

cudaError_t launch_delay_table_window(const double* delays, const double* fileoffsets, const int* fftindex,
                                      int first, int nant, int nfft, int ld, int F, int maxoffset, double sampletime,
                                      const double* win, int spb, int* err, DelayEntry* tab, uint32_t* vbits,
                                      cudaStream_t st)
{
    if (win && !err) return cudaErrorInvalidValue;
    dim3 grid((ld + 127) / 128, nant);
    k_delay_table<<<grid, 128, 0, st>>>(delays, fileoffsets, fftindex, first, nfft, ld, F, maxoffset, sampletime,
                                        win, nant, spb, err, tab, vbits);
    return cudaGetLastError();
}

cudaError_t launch_counts(const uint32_t* vbits, int nant, int nwords, int* counts, cudaStream_t st)
{
    const int npairs = nant * (nant + 1) / 2;
    k_counts<<<npairs, 256, 0, st>>>(vbits, nant, nwords, counts);
    return cudaGetLastError();
}

cudaError_t launch_finalize(const float2* acc, int acc_layout, int nsig, int npol, int nant, int nchan, int nsb,
                            const int* counts, int normalize, float2* vis, cudaStream_t st)
{
    k_finalize<<<1184, 256, 0, st>>>(acc, acc_layout, nsig, npol, nant, nchan, nsb, counts, normalize, vis);
    return cudaGetLastError();
}

// Amplitude and phase of each visibility in place, as saveVisibilities prints them (kernel.c:594-596,
// vectorMagnitude / vectorPhase): |v| = sqrt(re^2 + im^2) with the two squares and their sum
// rounded separately (no fused multiply-add), phase = atan2(im, re) in radians.
__global__ void k_amp_phase(float2* __restrict__ v, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float2 z = v[i];
        v[i] = make_float2(sqrtf(__fadd_rn(__fmul_rn(z.x, z.x), __fmul_rn(z.y, z.y))), atan2f(z.y, z.x));
    }
}

cudaError_t launch_amp_phase(float2* vis, long long n, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    const long long blocks = (n + 255) / 256;
    k_amp_phase<<<(int)(blocks < 1184 ? blocks : 1184), 256, 0, st>>>(vis, n);
    return cudaGetLastError();
}

}  // namespace fx
