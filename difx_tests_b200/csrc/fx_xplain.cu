// fx_xplain.cu -- plain FP32 X stage (baseline cross-multiply-accumulate).
//
// For every channel c and signal pair i <= j:
//     acc[sb][pair(i,j)][c] += sum_t X[sb][i][t][c] * conj(X[sb][j][t][c])
// which is kernel.c:829-854 (ippsAddProduct of channelised[j] and the conjugated
// channelised[k]) generalised to all signal pairs incl. autos; the conjugation
// of kernel.c:557-568 is folded into the multiply.
//
// Register tiling: each thread owns an 8x8 block of signal pairs for one
// channel (64 complex FP32 accumulators, 256 FFMA per time sample).  A CTA
// covers CG channels x every upper-triangle 8x8 tile, so each spectrum value is
// read from HBM/L2 once.  Time blocks of TK samples are double-buffered in
// shared memory with cp.async; lanes of a warp are (CG channels) x (32/CG
// tiles), so the operand loads are broadcasts or conflict-free.
//
// Small jobs (few channels, few signals) give fewer CTAs than SMs; there the
// time axis is cut too: CTA (c, sb, seg) sums FFT slots of segment seg into
// its own partials, and k_xplain_reduce adds the segments to acc in segment
// order, so the result does not depend on which CTA ran first.
#include "fx_common.cuh"
#include "fx_kernels.h"

namespace fx {

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// acc[ii][jj] += sum over the TK FFTs of a stage of xi[ii] * conj(xj[jj]) for one 8 x 8 tile of
// signal pairs (kernel.c:829-854; the conjugation of kernel.c:557-568 folded in).  pi / pj point at
// FFT 0 of the tile's first row / column signal in the stage; signals are SK elements apart, FFTs
// TKS.  The operands of FFT tk + 1 are loaded while FFT tk's 256 FMAs run, so the shared-memory
// latency hides behind independent arithmetic at two warps per scheduler.
//
// Each complex multiply-accumulate is two packed FP32 FMAs (fma.rn.f32x2 on the (re, im) pair):
//   acc += (a.y, a.x) * (b.y, -b.y), then acc += (a.x, a.y) * (b.x, b.x)
// i.e. re += a.y b.y then a.x b.x, im += -a.x b.y then a.y b.x: the operations and their order
// of the scalar form fma(a.x, b.x, fma(a.y, b.y, re)), fma(a.y, b.x, fma(-a.x, b.y, im)), so
// the sums are bit-identical to it, at half the FMA instructions.
__device__ __forceinline__ void cmac2(float2& acc, float2 a, float2 asw, float2 bxx, float2 byn)
{
    acc = __ffma2_rn(asw, byn, acc);
    acc = __ffma2_rn(a, bxx, acc);
}

template <int TK, int SK, int TKS>
__device__ __forceinline__ void tile_fma(float2 (&acc)[8][8], const float2 (&a)[8], const float2 (&b)[8])
{
    float2 asw[8];
#pragma unroll
    for (int ii = 0; ii < 8; ii++) asw[ii] = make_float2(a[ii].y, a[ii].x);
#pragma unroll
    for (int jj = 0; jj < 8; jj++) {
        // the two FMAs of one accumulator eight instructions apart (the FMA latency hides behind
        // the other accumulators of the column)
        const float2 bxx = make_float2(b[jj].x, b[jj].x), byn = make_float2(b[jj].y, -b[jj].y);
#pragma unroll
        for (int ii = 0; ii < 8; ii++) acc[ii][jj] = __ffma2_rn(asw[ii], byn, acc[ii][jj]);
#pragma unroll
        for (int ii = 0; ii < 8; ii++) acc[ii][jj] = __ffma2_rn(a[ii], bxx, acc[ii][jj]);
    }
}

template <int SK>
__device__ __forceinline__ void load8(float2 (&a)[8], float2 (&b)[8], const float2* pi, const float2* pj, int off)
{
#pragma unroll
    for (int k = 0; k < 8; k++) {
        a[k] = pi[off + k * SK];
        b[k] = pj[off + k * SK];
    }
}

// acc[ii][jj] += sum over the TK FFTs of a stage of xi[ii] * conj(xj[jj]) for one 8 x 8 tile of
// signal pairs (kernel.c:829-854; the conjugation of kernel.c:557-568 folded in).  pi / pj point at
// FFT 0 of the tile's first row / column signal in the stage; signals are SK elements apart, FFTs
// TKS.  Two operand sets alternate: the operands of FFT tk + 1 are loaded while FFT tk's 256 FMAs
// run (no register copies between them), so the shared-memory latency hides behind independent
// arithmetic at two warps per scheduler.
template <int TK, int SK, int TKS>
__device__ __forceinline__ void tile_stage(float2 (&acc)[8][8], const float2* pi, const float2* pj)
{
    static_assert(TK % 2 == 0, "FFTs of a stage in pairs");
    float2 a0[8], b0[8], a1[8], b1[8];
    load8<SK>(a0, b0, pi, pj, 0);
#pragma unroll 1
    for (int tk = 0; tk < TK; tk += 2) {
        load8<SK>(a1, b1, pi, pj, (tk + 1) * TKS);
        tile_fma<TK, SK, TKS>(acc, a0, b0);
        if (tk + 2 < TK) load8<SK>(a0, b0, pi, pj, (tk + 2) * TKS);
        tile_fma<TK, SK, TKS>(acc, a1, b1);
    }
}

// The upper triangles (ii <= jj, index jj (jj + 1) / 2 + ii) of two diagonal 8 x 8 blocks, A at
// pa and B at pb: 72 pairs, the work of one tile, with the same alternating operand sets.
__device__ __forceinline__ void diag_fma(float2 (&acc)[2][36], const float2 (&a)[8], const float2 (&b)[8])
{
    float2 asw[8], bsw[8];
#pragma unroll
    for (int ii = 0; ii < 8; ii++) {
        asw[ii] = make_float2(a[ii].y, a[ii].x);
        bsw[ii] = make_float2(b[ii].y, b[ii].x);
    }
#pragma unroll
    for (int jj = 0; jj < 8; jj++) {
        const float2 axx = make_float2(a[jj].x, a[jj].x), ayn = make_float2(a[jj].y, -a[jj].y);
        const float2 bxx = make_float2(b[jj].x, b[jj].x), byn = make_float2(b[jj].y, -b[jj].y);
#pragma unroll
        for (int ii = 0; ii <= jj; ii++) {
            cmac2(acc[0][jj * (jj + 1) / 2 + ii], a[ii], asw[ii], axx, ayn);
            cmac2(acc[1][jj * (jj + 1) / 2 + ii], b[ii], bsw[ii], bxx, byn);
        }
    }
}

template <int TK, int SK, int TKS>
__device__ __forceinline__ void diag_pair_stage(float2 (&acc)[2][36], const float2* pa, const float2* pb)
{
    float2 a0[8], b0[8], a1[8], b1[8];
    load8<SK>(a0, b0, pa, pb, 0);
#pragma unroll 1
    for (int tk = 0; tk < TK; tk += 2) {
        load8<SK>(a1, b1, pa, pb, (tk + 1) * TKS);
        diag_fma(acc, a0, b0);
        if (tk + 2 < TK) load8<SK>(a0, b0, pa, pb, (tk + 2) * TKS);
        diag_fma(acc, a1, b1);
    }
}

// Plan of one channel group: NB blocks of 8 signals.  With NB = 8 the 36 upper 8 x 8 tiles are
// re-cut as 28 off-diagonal tiles plus 4 threads that each take the upper triangles of two
// diagonal blocks (b, 7 - b): 32 equal threads per channel, so 8 channels fill 8 warps and each
// thread keeps the registers for the prefetched operands (a scheduler's register file is shared
// by its warps; 9 warps would leave 168 per thread).  With NB = 4 the same cut gives 6 + 2 = 8
// equal threads per channel instead of 10 (4 of them half idle on diagonal tiles): 32 channels
// fill 8 warps, again with the prefetch.
template <int NB, int CG, int TK>
struct XPlan {
    static constexpr bool PAIRED = NB == 8 || NB == 4;
    static constexpr int NOFF = NB * (NB - 1) / 2;
    static constexpr int NTILE = PAIRED ? NOFF + NB / 2 : NB * (NB + 1) / 2;
    static constexpr int NTHREADS = CG * NTILE;
    static constexpr bool PIPE = NTHREADS <= 256;           // prefetch only where the registers allow
    static constexpr int NS = NB * 8;                       // staged signals
    // element (s, tk, cl) at s*TK*CG + (s/8)*8 + tk*CG + cl  (64-byte skew per 8-signal block)
    static constexpr int STAGE = NS * TK * CG + NB * 8;     // float2 per buffer
};

template <int NB, int CG, int TK>
__device__ __forceinline__ int xoff(int s, int tk, int cl)
{
    return s * TK * CG + (s >> 3) * 8 + tk * CG + cl;
}

// Stages of one X-stage block for one thread: tiles (DP false) or diagonal pairs (DP true).
template <int NB, int CG, int TK, bool DP>
__device__ __forceinline__ void xplain_stages(const XArgs& a, int sb, int c0, float2* xs, int tid, int cl, int I,
                                              int J, int seg)
{
    using P = XPlan<NB, CG, TK>;
    const int nsig = a.nsig;
    const int C = a.nchan;
    const float2* spec = reinterpret_cast<const float2*>(a.spec) + (size_t)sb * nsig * a.T * C;

    // zero the padding signals once (both buffers)
    for (int e = tid; e < 2 * P::STAGE; e += P::NTHREADS) xs[e] = make_float2(0.f, 0.f);
    __syncthreads();

    constexpr int VPR = CG / 2;                                    // 16-byte vectors per (s, tk) row
    const int nvec = nsig * TK * VPR;
    auto issue = [&](int buf, int t0) {
        float2* dst = xs + buf * P::STAGE;
        for (int v = tid; v < nvec; v += P::NTHREADS) {
            const int s = v / (TK * VPR);
            const int r = v - s * (TK * VPR);
            const int tk = r / VPR;
            const int q = r - tk * VPR;
            const float2* src = spec + ((size_t)s * a.T + t0 + tk) * C + c0 + 2 * q;
            cp_async16(dst + xoff<NB, CG, TK>(s, tk, 2 * q), src);
        }
        cp_async_commit();
    };

    // DP: upper triangles of diagonal blocks I and J; otherwise the I x J tile
    float2 acc[DP ? 1 : 8][8];
    float2 dacc[DP ? 2 : 1][36];
#pragma unroll
    for (int i = 0; i < (DP ? 1 : 8); i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = make_float2(0.f, 0.f);
#pragma unroll
    for (int h = 0; h < (DP ? 2 : 1); h++)
#pragma unroll
        for (int i = 0; i < 36; i++) dacc[h][i] = make_float2(0.f, 0.f);

    // FFT slots [t_lo, t_hi): all of them, or segment seg of tlen slots (an empty segment adds zeros)
    const int nslot = a.ntk ? a.ntk : a.T;
    const bool segd = a.tseg > 1;
    const int t_lo = segd ? min(seg * a.tlen, nslot) : 0;
    const int t_hi = segd ? min(t_lo + a.tlen, nslot) : nslot;
    const int nblk = (t_hi - t_lo) / TK;
    if (nblk > 0) issue(0, t_lo);
    for (int blk = 0; blk < nblk; blk++) {
        if (blk + 1 < nblk) {
            issue((blk + 1) & 1, t_lo + (blk + 1) * TK);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const float2* x = xs + (blk & 1) * P::STAGE;
        // within a block of 8 signals the skew is constant: signal s + k is k * TK * CG further
        const float2* pi = x + xoff<NB, CG, TK>(I * 8, 0, cl);
        const float2* pj = x + xoff<NB, CG, TK>(J * 8, 0, cl);
        if constexpr (DP) {
            diag_pair_stage<TK, TK * CG, CG>(dacc, pi, pj);
        } else if constexpr (P::PIPE) {
            tile_stage<TK, TK * CG, CG>(acc, pi, pj);
        } else {
            // one operand set at a time (no prefetch: more than 256 threads leave no registers for
            // a second set), the same packed FMAs
            for (int tk = 0; tk < TK; tk++) {
                float2 xi[8], xj[8];
                load8<TK * CG>(xi, xj, pi, pj, tk * CG);
                tile_fma<TK, TK * CG, CG>(acc, xi, xj);
            }
        }
        __syncthreads();   // buffer (blk & 1) is refilled by the next issue
    }

    float2* out = reinterpret_cast<float2*>(a.acc);
    const int npair = nsig * (nsig + 1) / 2;
    // this segment's partial sums: [seg][sb][pair][chan], the layout of acc per segment
    float2* part = segd ? reinterpret_cast<float2*>(a.part) + (size_t)seg * a.nsb * npair * C : nullptr;
    if constexpr (DP) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int B = h ? J : I;
#pragma unroll
            for (int jj = 0; jj < 8; jj++)
#pragma unroll
                for (int ii = 0; ii <= jj; ii++) {
                    const int i = B * 8 + ii, j = B * 8 + jj;
                    if (j < nsig) {
                        const int p = i * nsig - (i * (i - 1)) / 2 + (j - i);
                        const size_t e = ((size_t)sb * npair + p) * C + c0 + cl;
                        const float2 v = dacc[h][jj * (jj + 1) / 2 + ii];
                        if (segd) {
                            part[e] = v;
                        } else {
                            float2 cur = out[e];
                            cur.x += v.x;
                            cur.y += v.y;
                            out[e] = cur;
                        }
                    }
                }
        }
    } else {
#pragma unroll
        for (int ii = 0; ii < 8; ii++) {
            const int i = I * 8 + ii;
#pragma unroll
            for (int jj = 0; jj < 8; jj++) {
                const int j = J * 8 + jj;
                if (i <= j && j < nsig) {
                    const int p = i * nsig - (i * (i - 1)) / 2 + (j - i);
                    const size_t e = ((size_t)sb * npair + p) * C + c0 + cl;
                    if (segd) {
                        part[e] = acc[ii][jj];
                    } else {
                        float2 cur = out[e];
                        cur.x += acc[ii][jj].x;
                        cur.y += acc[ii][jj].y;
                        out[e] = cur;
                    }
                }
            }
        }
    }
}

// One X-stage block: channels [c0, c0 + CG) of subband sb over all T FFT slots.
template <int NB, int CG, int TK>
__device__ __forceinline__ void xplain_block(const XArgs& a, int sb, int c0, int seg, unsigned char* smem)
{
    using P = XPlan<NB, CG, TK>;
    float2* xs = reinterpret_cast<float2*>(smem);   // [2][STAGE]

    const int tid = threadIdx.x;
    const int tile = tid / CG;
    const int cl = tid - tile * CG;
    // tile -> block pair (I, J): off-diagonal I < J first when PAIRED, else the upper triangle I <= J;
    // PAIRED tiles NOFF.. are diagonal pairs (I, NB - 1 - I) (whole warps: warp-uniform branches)
    const bool dpair = P::PAIRED && tile >= P::NOFF;
    int I = 0, J = 0;
    if (dpair) {
        I = tile - P::NOFF;
        J = NB - 1 - I;
    } else {
        const int lead = P::PAIRED ? 1 : 0;   // off-diagonal rows hold NB - 1 - I tiles
        int rem = tile;
        while (rem >= NB - lead - I) {
            rem -= NB - lead - I;
            I++;
        }
        J = I + lead + rem;
    }

    // the two thread kinds in separate instantiations, so each keeps only its own accumulators
    if (dpair)
        xplain_stages<NB, CG, TK, true>(a, sb, c0, xs, tid, cl, I, J, seg);
    else
        xplain_stages<NB, CG, TK, false>(a, sb, c0, xs, tid, cl, I, J, seg);
}

template <int NB, int CG, int TK>
__global__ void __launch_bounds__(XPlan<NB, CG, TK>::NTHREADS, 1)
k_xplain(XArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    xplain_block<NB, CG, TK>(a, blockIdx.y, blockIdx.x * CG, blockIdx.z, smem);
}

// Many jobs with the same tile plan in one launch: CTA i takes task i {job, subband, first
// channel} of the table, and the hardware's block scheduler balances the uneven jobs over the
// SMs (a persistent grid striding over the table measured 13 % slower on the 12-job batch).
template <int NB, int CG, int TK>
__global__ void __launch_bounds__(XPlan<NB, CG, TK>::NTHREADS, 1)
k_xplain_batch(const XArgs* __restrict__ jobs, const int4* __restrict__ tasks, int ntask)
{
    extern __shared__ __align__(16) unsigned char smem[];
    if (blockIdx.x < ntask) {
        const int4 tk = tasks[blockIdx.x];
        const XArgs& a = jobs[tk.x];   // read where used (global, cached)
        xplain_block<NB, CG, TK>(a, tk.y, tk.z, tk.w, smem);
    }
}

template <int NB, int CG, int TK>
static cudaError_t launch_x(const XArgs& a, cudaStream_t st)
{
    using P = XPlan<NB, CG, TK>;
    if (a.nchan % CG) return cudaErrorInvalidValue;
    const size_t sm = 2 * (size_t)P::STAGE * sizeof(float2);
    auto kern = k_xplain<NB, CG, TK>;
    static unsigned configured = 0;  // per instantiation and device
    cudaError_t e = set_smem_once(kern, sm, &configured);
    if (e != cudaSuccess) return e;
    const int tseg = xplain_segments_used(a);
    if (a.tseg > 1 && !a.part) return cudaErrorInvalidValue;
    dim3 grid(a.nchan / CG, a.nsb, tseg);
    kern<<<grid, P::NTHREADS, sm, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return a.tseg > 1 ? launch_xplain_reduce(a, st) : cudaSuccess;
}

template <int NB, int CG, int TK>
static cudaError_t launch_xb(const XArgs* d_jobs, const int4* d_tasks, int ntask, cudaStream_t st)
{
    using P = XPlan<NB, CG, TK>;
    const size_t sm = 2 * (size_t)P::STAGE * sizeof(float2);
    auto kern = k_xplain_batch<NB, CG, TK>;
    static unsigned configured = 0;
    cudaError_t e = set_smem_once(kern, sm, &configured);
    if (e != cudaSuccess) return e;
    if (ntask <= 0) return cudaSuccess;
    kern<<<ntask, P::NTHREADS, sm, st>>>(d_jobs, d_tasks, ntask);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------
// More than 64 signals: the signal range is cut into super-blocks of 64 and a CTA
// owns one super-block pair (P, Q), P <= Q, for CG channels: 8 x 8 register
// tiles of 8 x 8 signal pairs, one per thread and channel (tiles below the
// diagonal of a diagonal pair idle).  Both super-blocks are staged per TK FFTs.
namespace big {
constexpr int CG = 4;            // channels per CTA
constexpr int TK = 16;           // FFTs per stage
constexpr int NTHREADS = 64 * CG;
constexpr int NS = 128;          // staged signals: 64 rows (P) + 64 columns (Q)
// element (s, tk, cl) at s*TK*CG + (s/8)*4 + tk*CG + cl: the 4-element skew per 8 signals
// spreads the column operands of a warp's 8 tiles over the banks (2 wavefronts per load)
constexpr int STAGE = NS * TK * CG + (NS / 8) * 4;
__device__ __forceinline__ int off(int s, int tk, int cl) { return s * TK * CG + (s >> 3) * 4 + tk * CG + cl; }
}  // namespace big

__device__ __forceinline__ void super_pair(int bp, int nb, int& P, int& Q)
{
    P = 0;
    while (bp >= nb - P) {
        bp -= nb - P;
        P++;
    }
    Q = P + bp;
}

__global__ void __launch_bounds__(big::NTHREADS, 1)
k_xplain_big(XArgs a)
{
    using namespace big;
    extern __shared__ __align__(16) unsigned char smem[];
    float2* xs = reinterpret_cast<float2*>(smem);   // [2][STAGE]
    const int sb = blockIdx.z;
    const int c0 = blockIdx.x * CG;
    const int nsig = a.nsig;
    const int nsup = (nsig + 63) / 64;
    int P, Q;
    super_pair(blockIdx.y, nsup, P, Q);

    const int tid = threadIdx.x;
    const int tile = tid / CG;
    const int cl = tid - tile * CG;
    const int ti = tile >> 3, tj = tile & 7;
    const bool active = !(P == Q && ti > tj);

    const int C = a.nchan;
    const float2* spec = reinterpret_cast<const float2*>(a.spec) + (size_t)sb * nsig * a.T * C;

    for (int e = tid; e < 2 * STAGE; e += NTHREADS) xs[e] = make_float2(0.f, 0.f);
    __syncthreads();

    constexpr int VPR = CG / 2;   // 16-byte vectors per (s, tk)
    auto issue = [&](int buf, int t0) {
        float2* dst = xs + buf * STAGE;
        for (int v = tid; v < NS * TK * VPR; v += NTHREADS) {
            const int s = v / (TK * VPR);
            const int r = v - s * (TK * VPR);
            const int tk = r / VPR;
            const int q = r - tk * VPR;
            const int sig = (s < 64) ? P * 64 + s : Q * 64 + (s - 64);
            if (sig < nsig) {
                const float2* src = spec + ((size_t)sig * a.T + t0 + tk) * C + c0 + 2 * q;
                cp_async16(dst + off(s, tk, 2 * q), src);
            }
        }
        cp_async_commit();
    };

    float2 acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = make_float2(0.f, 0.f);

    const int nblk = (a.ntk ? a.ntk : a.T) / TK;
    issue(0, 0);
    for (int blk = 0; blk < nblk; blk++) {
        if (blk + 1 < nblk) {
            issue((blk + 1) & 1, (blk + 1) * TK);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const float2* x = xs + (blk & 1) * STAGE;
        // 256 threads: two warps per scheduler, registers for the prefetched operands
        if (active) tile_stage<TK, TK * CG, CG>(acc, x + off(ti * 8, 0, cl), x + off(64 + tj * 8, 0, cl));
        __syncthreads();
    }
    if (!active) return;
    float2* out = reinterpret_cast<float2*>(a.acc);
    const size_t npair = (size_t)nsig * (nsig + 1) / 2;
#pragma unroll
    for (int ii = 0; ii < 8; ii++) {
        const int i = P * 64 + ti * 8 + ii;
#pragma unroll
        for (int jj = 0; jj < 8; jj++) {
            const int j = Q * 64 + tj * 8 + jj;
            if (i <= j && j < nsig) {
                const size_t p = (size_t)i * nsig - ((size_t)i * (i - 1)) / 2 + (j - i);
                float2* o = out + ((size_t)sb * npair + p) * C + c0 + cl;
                float2 cur = *o;
                cur.x += acc[ii][jj].x;
                cur.y += acc[ii][jj].y;
                *o = cur;
            }
        }
    }
}

static cudaError_t launch_xbig(const XArgs& a, cudaStream_t st)
{
    if (a.nchan % big::CG || a.T % big::TK || a.ntk % big::TK || a.ntk > a.T || a.nsig > 512)
        return cudaErrorInvalidValue;
    const size_t sm = 2 * (size_t)big::STAGE * sizeof(float2);
    static unsigned configured = 0;
    cudaError_t e = set_smem_once(k_xplain_big, sm, &configured);
    if (e != cudaSuccess) return e;
    const int nsup = (a.nsig + 63) / 64;
    dim3 grid(a.nchan / big::CG, nsup * (nsup + 1) / 2, a.nsb);
    k_xplain_big<<<grid, big::NTHREADS, sm, st>>>(a);
    return cudaGetLastError();
}

// Tile plans per signal count: NB = ceil(nsig/8) blocks of 8 signals; CG
// channels per CTA and TK FFTs per shared-memory stage.  Variant 0 is the
// built-in choice, variant 1 the alternative the autotuner may pick.
#define FX_XPLANS(OP)                                                           \
    switch (nb * 2 + (alt ? 1 : 0)) {                                           \
    case 2: OP(1, 32, 8); case 3: OP(1, 16, 16);                                \
    case 4: OP(2, 32, 8); case 5: OP(2, 16, 16);                                \
    case 6: OP(3, 32, 8); case 7: OP(3, 16, 16);                                \
    case 8: OP(4, 32, 8); case 9: OP(4, 16, 16);                                \
    case 10: OP(5, 16, 8); case 11: OP(5, 8, 16);                               \
    case 12: OP(6, 16, 8); case 13: OP(6, 8, 16);                               \
    case 14: OP(7, 8, 16); case 15: OP(7, 8, 8);                                \
    case 16: OP(8, 8, 16); case 17: OP(8, 8, 8);                                \
    default: return cudaErrorNotSupported;                                      \
    }

// acc[e] += (part[0][e] + part[1][e] + ... + part[tseg - 1][e]), summed in segment order
__global__ void k_xplain_reduce(float2* __restrict__ acc, const float2* __restrict__ part, int tseg, long long n)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        float2 s = part[e];
        for (int t = 1; t < tseg; t++) {
            const float2 v = part[t * n + e];
            s.x += v.x;
            s.y += v.y;
        }
        float2 cur = acc[e];
        cur.x += s.x;
        cur.y += s.y;
        acc[e] = cur;
    }
}

// Segments a launch computes: those holding slots below ntk (later ones would only add zeros)
int xplain_segments_used(const XArgs& a)
{
    if (a.tseg <= 1) return 1;
    const int nslot = a.ntk ? a.ntk : a.T;
    return std::max(1, std::min(a.tseg, (nslot + a.tlen - 1) / a.tlen));
}

cudaError_t launch_xplain_reduce(const XArgs& a, cudaStream_t st)
{
    if (a.tseg <= 1) return cudaSuccess;
    const long long n = (long long)a.nsb * (a.nsig * (a.nsig + 1) / 2) * a.nchan;
    const long long blocks = (n + 255) / 256;
    k_xplain_reduce<<<(int)(blocks < 1184 ? blocks : 1184), 256, 0, st>>>(
        reinterpret_cast<float2*>(a.acc), reinterpret_cast<const float2*>(a.part), xplain_segments_used(a), n);
    return cudaGetLastError();
}

// CTAs of the plain X kernel of nsig signals and tile variant alt resident on one SM
template <int NB, int CG, int TK>
static cudaError_t occ_x(int* per_sm)
{
    using P = XPlan<NB, CG, TK>;
    const size_t sm = 2 * (size_t)P::STAGE * sizeof(float2);
    auto kern = k_xplain<NB, CG, TK>;
    static unsigned configured = 0;
    cudaError_t e = set_smem_once(kern, sm, &configured);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern, P::NTHREADS, sm);
}

static cudaError_t xplain_occupancy(int nsig, int alt, int* per_sm)
{
    const int nb = (nsig + 7) / 8;
#define FX_OP(NB_, CG_, TK_) return occ_x<NB_, CG_, TK_>(per_sm)
    FX_XPLANS(FX_OP)
#undef FX_OP
}

// Time segments of the plain X stage (up to 64 signals).  With C CTAs of channel groups (default
// tile variant) and R = SMs x resident CTAs of its kernel, cutting the T FFT slots into s segments
// of L = ceil(T / s) slots (a multiple of 16, at least 64) takes about ceil(C s / R) waves of L + 32
// slots each (32: a CTA's fixed cost, its first stage load and its partial sums); the s of the
// least time is taken, up to 32 (s = 1: no segments, the CTAs add to the accumulators).  A
// function of the job's geometry and the device only (not of the tile variant), so a batch and the
// single-job path cut a job the same way and sum it in the same order, tuned or not.
void xplain_segment_model(long long ctas, long long slots, int T, int* tseg, int* tlen)
{
    *tseg = 1;
    *tlen = T;
    if (ctas < 1 || slots < 1 || T < 128) return;
    auto cost = [&](int len) {
        const long long nseg = (T + len - 1) / len;
        return ((ctas * nseg + slots - 1) / slots) * (long long)(len + 32);
    };
    int best_len = T;
    long long best = cost(T);
    for (int sg = 2; sg <= 32; sg++) {
        const int len = ((T + sg - 1) / sg + 15) / 16 * 16;
        if (len < 64) break;
        const long long c = cost(len);
        if (c < best) {
            best = c;
            best_len = len;
        }
    }
    if (best_len >= T) return;
    *tlen = best_len;
    *tseg = (T + best_len - 1) / best_len;
}

void xplain_segments(int nsig, int nchan, int nsb, int T, int nsm, int* tseg, int* tlen)
{
    *tseg = 1;
    *tlen = T;
    if (nsig > 64 || nsig < 1 || T < 128) return;
    const long long ctas = (long long)(nchan / xplain_channel_group(nsig, 0)) * nsb;
    int occ = 0;
    if (xplain_occupancy(nsig, 0, &occ) != cudaSuccess || occ < 1) {
        (void)cudaGetLastError();
        occ = 1;
    }
    xplain_segment_model(ctas, (long long)nsm * occ, T, tseg, tlen);
}

int xplain_channel_group(int nsig, int alt)
{
    const int nb = (nsig + 7) / 8;
#define FX_CG(NB_, CG_, TK_) return CG_
    switch (nb * 2 + (alt ? 1 : 0)) {
    case 2: case 4: case 6: case 8: FX_CG(0, 32, 0);
    case 3: case 5: case 7: case 9: case 10: case 12: FX_CG(0, 16, 0);
    default: FX_CG(0, 8, 0);
    }
#undef FX_CG
}

cudaError_t launch_xplain(const XArgs& a, cudaStream_t st)
{
    if (a.nsig > 64) return launch_xbig(a, st);
    const int nb = (a.nsig + 7) / 8;
    const int alt = a.alt;
    if (a.T % 16 != 0 || a.ntk % 16 != 0 || a.ntk > a.T) return cudaErrorInvalidValue;  // multiples of every TK
#define FX_OP(NB_, CG_, TK_) return launch_x<NB_, CG_, TK_>(a, st)
    FX_XPLANS(FX_OP)
#undef FX_OP
}

cudaError_t launch_xplain_batch(int nsig, int alt, const XArgs* d_jobs, const int4* d_tasks, int ntask,
                                cudaStream_t st)
{
    const int nb = (nsig + 7) / 8;
#define FX_OP(NB_, CG_, TK_) return launch_xb<NB_, CG_, TK_>(d_jobs, d_tasks, ntask, st)
    FX_XPLANS(FX_OP)
#undef FX_OP
}

}  // namespace fx
