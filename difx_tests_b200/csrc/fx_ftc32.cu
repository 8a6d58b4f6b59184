// fx_ftc32.cu -- FP32-grade tensor-core F stage for 2048-point FFTs (1024 channels) of one
// polarisation of 2-bit real input.
//
// The same 32 x 64 split of the DFT as the FP16 tensor-core F stage (fx_ftc.cu), along the
// factorisation the reference's rotators use (kernel.c:31-36, 160-165), with sample
// n = 64 n1 + n2 and channel k = k1 + 32 k2:
//   X[k1 + 32 k2] = fstep[k2] sum_n2 W64^(n2 k2) [sub[n2] W2048^(n2 k1) fsub[k1]] sum_n1 W32^(n1 k1) x[n]
// with x[n] = level(n) step[n1] (the fringe rotator is sub[n2] step[n1], kernel.c:428-497, and
// the fractional-sample rotator of channel k is fsub[k1] fstep[k2], kernel.c:512-555).  Every
// FP16 operand is an error-compensated pair hi + lo (hi = FP16 rounding of the FP32 value,
// lo = FP16 rounding of the remainder) and each GEMM accumulates the three products
// hi.hi + lo.hi + hi.lo in FP32 TMEM: the spectra carry FP32-level error (~2e-7 of max|X|),
// not FP16-level (~3e-4).
//   step 1   D1[(b, n2)][(k1, re|im)] = A1 . B1^T, A1 = x in TMEM, M128 N64 K64, x3 products
//            (A1 comes from a per-(FFT, n1) table of the four levels times step[n1]: exact pairs)
//   twiddle  Z = D1 * sub[n2] W2048^(n2 k1) fsub[k1] on the CUDA cores (FP32; the factor is
//            e^{i alpha k1} times sub[n2], a complex recurrence over k1 restarted at k1 = 16)
//   step 2   D2[(k1 % 16, b)][(k2, re|im)] = A2 . B2^T, A2 = Z in shared memory, M128 N64 K128,
//            x3 products, k2 < 32 (channels < 1024)
//   output   X = D2 * fstep[k2] -> FP16 K-major spectra (tensor-core X forms; for the FP8 form also
//            the absmax of each (channel, signal) over the chunk) or FP32 channel-contiguous
//            spectra (plain form and the spectra check)
// b = the FFT within a work item of 8 consecutive FFTs of one (subband, antenna).
//
// Persistent, warp-specialised CTA (one per SM, 736 threads):
//   warps 0-3    producer: 2-bit codes -> table lookups -> A1 pairs (TMEM, two stages)
//   warps 4-11   twiddle: D1 (TMEM, one slot per pair of the item) -> Z pairs -> A2 (shared);
//                tile 0 (k1 < 16) for the item's four pairs, then tile 1, so the step-2 MMAs
//                of one tile run while the other is written; also the item's fstep table
//   warps 12-19  output, two groups of four: D2 (TMEM, one slot per tile; group g takes
//                columns 32 g .. 32 g + 31) -> fstep -> an FP16 box per warp in shared memory
//                written out by one tensor store (or FP32 spectra by plain stores)
//   warp 20      MMA issuer (one elected lane), TMEM owner
//   warps 21-22  helpers (alternate pairs): up to four pairs ahead, the input bulk copies, the
//                level x step tables and the window offsets
// 23 warps are 6 on three of the four schedulers, which holds every thread to 80 registers.
// Every wait is bounded (1 s): on expiry the CTA records code 7 in the error word, stops,
// drains what it issued and frees TMEM (or keeps it allocated if the drain itself expires).
#include <cstring>

#include "fx_ftc_common.cuh"

namespace fx {
namespace ftc32 {

using namespace ftcc;
using P = FPlan<2048>;
constexpr int C = P::C;                   // 1024 channels
constexpr int F1 = P::STRIDE;             // 32: n1, k1
constexpr int F2 = P::S;                  // 64: n2
constexpr int K2H = C / F1;               // 32: k2 of the kept channels
static_assert(F1 == 32 && F2 == 64 && K2H == 32 && P::FS == F1 && P::FST == K2H, "2048-point split");
constexpr int TB = 8;                     // FFTs per work item
constexpr int NPAIR = TB / 2;             // step-1 tiles (FFT pairs) per item
constexpr int NA1 = 2;                    // A1 stages (TMEM)
constexpr int NIB = 4;                    // pair slots the helper fills ahead of the producer
constexpr int NOUT = 8;                   // output warps (two per TMEM lane quarter)
constexpr int NHELP = 2;                  // helper warps (alternate pairs)
constexpr int NTHREADS = 736;             // 23 warps
constexpr int W_TW = 4, W_OUT = 12, W_MMA = W_OUT + NOUT, W_HELP = W_MMA + 1;
constexpr uint32_t TMEM_COLS = 512;
constexpr uint32_t A1_COL = 0;            // [stage] 64 columns: x_hi (n1, re|im) | x_lo
constexpr uint32_t D1_COL = 128;          // [pair of the item] 64 columns (k1, re|im)
constexpr uint32_t D2_COL = 384;          // [tile] 64 columns (k2, re|im)
constexpr int ERR_WAIT = 7;
constexpr uint32_t kIdesc = tc::idesc_f16(128, 64);

struct Smem {
    alignas(1024) uint8_t a2[2][2][2][128 * 128];   // [tile][hi|lo][K half] rows 8 (k1 % 16) + b, (n2 % 32, re|im)
    alignas(1024) uint8_t b1[2][64 * 128];          // [hi|lo] rows (k1, re|im), K (n1, re|im)
    alignas(1024) uint8_t b2[2][2][64 * 128];       // [hi|lo][K half] rows (k2, re|im), K (n2 % 32, re|im)
    alignas(16) uint8_t inb[NIB][2][INB];           // [pair % NIB][FFT of the pair] input bytes
    alignas(16) uint2 lut[NIB][2][F1][4];           // [pair % NIB][FFT][n1][code] (hi, lo) of level * step[n1]
    int2 pwin[NIB][2];                              // [pair % NIB][FFT] (bit of sample 0 in inb, valid)
    float2 fstep[2][K2H][TB];                       // [item parity][k2][b] fstep of the item's FFTs (a warp's
                                                    // 8 FFTs: one 64-byte row), written by the twiddle warps
    alignas(128) __half otile[NOUT][2][16 * 4 * 2 * TB]; // output: [warp][buffer] FP16 boxes
                                                          // [k2 % 16][k1 % 4][re|im][b] of the tensor store
    float ctab[P::FS + P::FST];                     // chan_sub | chan_step
    uint64_t a1_full[NA1], a1_empty[NA1], d1_full[NPAIR], d1_empty[NPAIR];
    uint64_t a2_full[2], a2_empty[2], d2_full[2], d2_empty[2], drain;
    uint64_t cp_full[NIB], tab_full[NIB], tab_empty[NIB];
    uint64_t fs_full[2], fs_empty[2];
    uint32_t tmem_base;
    int abort;
    int drain_fail;                                 // a drain wait expired: copies or MMAs may be in flight
};
static_assert(sizeof(Smem) + 1024 <= 232448, "fits the opt-in shared memory of one CTA");

// FP16 pair (hi, lo) of an FP32 complex value, each packed (re, im)
__device__ __forceinline__ uint2 split_pair(float re, float im)
{
    const __half2 hi = __floats2half2_rn(re, im);
    const float2 hf = __half22float2(hi);
    const __half2 lo = __floats2half2_rn(re - hf.x, im - hf.y);
    return make_uint2(h2u(hi), h2u(lo));
}

// The same pair with hi = v truncated to 11 significant bits (sign, exponent and the top 10
// fraction bits kept): hi is exact in FP16 (to 2^-25 absolute below FP16's normal range), lo =
// RN16(v - hi) with v - hi exact in FP32; together ~21 bits.  No FP16 -> FP32 conversions.
__device__ __forceinline__ uint2 split_pair_t(float re, float im)
{
    const float hr = __uint_as_float(__float_as_uint(re) & 0xFFFFE000u);
    const float hm = __uint_as_float(__float_as_uint(im) & 0xFFFFE000u);
    return make_uint2(h2u(__floats2half2_rn(hr, hm)), h2u(__floats2half2_rn(re - hr, im - hm)));
}

// e^{i a} for |a| <= 0.25 by its Taylor series to the a^8 / a^9 terms (truncation < 1e-10)
__device__ __forceinline__ float2 cis_small(float a)
{
    const float a2 = a * a;
    const float c = 1.f - a2 * (0.5f - a2 * (1.f / 24.f - a2 * (1.f / 720.f - a2 * (1.f / 40320.f))));
    const float s = a * (1.f - a2 * (1.f / 6.f - a2 * (1.f / 120.f - a2 * (1.f / 5040.f - a2 * (1.f / 362880.f)))));
    return make_float2(c, s);
}

__device__ __forceinline__ float2 cis_half_turns_acc(float x)
{
    float s, c;
    sincospif(x, &s, &c);
    return make_float2(c, s);
}

template <bool OUT16, bool AMAX>
__global__ void __launch_bounds__(NTHREADS, 1) k_ftc32(FArgs a, const __grid_constant__ CUtensorMap omap)
{
    using namespace tc;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    Smem& sm = *reinterpret_cast<Smem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    volatile int* abort_flag = &sm.abort;

    const int tspan = a.tspan ? a.tspan : a.T;
    const int ntb = tspan / TB;
    const int ntask = a.nsb * a.nant * ntb;
    const int nitem = blockIdx.x < ntask ? (ntask - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    // ---- set-up: barriers, TMEM, constant DFT matrices (hi, lo), channel table
    if (threadIdx.x == 0) {
        for (int s = 0; s < NA1; s++) {
            mbar_init(&sm.a1_full[s], 128);
            mbar_init(&sm.a1_empty[s], 1);
        }
        for (int p = 0; p < NPAIR; p++) {
            mbar_init(&sm.d1_full[p], 1);
            mbar_init(&sm.d1_empty[p], 128);
        }
        for (int j = 0; j < 2; j++) {
            mbar_init(&sm.a2_full[j], 256);
            mbar_init(&sm.a2_empty[j], 1);
            mbar_init(&sm.d2_full[j], 1);
            mbar_init(&sm.d2_empty[j], 32 * NOUT);
        }
        mbar_init(&sm.drain, 1);
        for (int s = 0; s < 2; s++) {
            mbar_init(&sm.fs_full[s], 256);
            mbar_init(&sm.fs_empty[s], 32 * NOUT);
        }
        for (int s = 0; s < NIB; s++) {
            mbar_init(&sm.cp_full[s], 1);
            mbar_init(&sm.tab_full[s], 1);
            mbar_init(&sm.tab_empty[s], 128);
        }
        sm.abort = 0;
        sm.drain_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == W_MMA) tmem_alloc(&sm.tmem_base, TMEM_COLS);
    // B1[(k1, c)][(n1, c')] and B2[(k2, c)][(n2, c')]: real form of W^(n k), w = (Re, Im) of W:
    // (c, c') = (0, 0) Re, (0, 1) -Im, (1, 0) Im, (1, 1) Re; each entry as an FP16 pair
    for (int e = threadIdx.x; e < 64 * 64 * 3; e += NTHREADS) {
        const int m = e / (64 * 64);          // 0: B1, 1-2: B2 K halves
        const int rem = e - m * 64 * 64;
        const int nb = rem >> 6, kk = rem & 63;
        const int c = nb & 1, cp = kk & 1;
        float2 w;
        uint8_t *hi, *lo;
        if (m == 0) {
            w = twiddle_exact(((kk >> 1) * (nb >> 1)) & (F1 - 1), F1);
            hi = sm.b1[0];
            lo = sm.b1[1];
        } else {
            const int n2 = (m - 1) * 32 + (kk >> 1);
            w = twiddle_exact((n2 * (nb >> 1)) & (F2 - 1), F2);
            hi = sm.b2[0][m - 1];
            lo = sm.b2[1][m - 1];
        }
        const float v = c == 0 ? (cp == 0 ? w.x : -w.y) : (cp == 0 ? w.y : w.x);
        const __half h = __float2half_rn(v);
        const uint32_t o = sw128(nb, kk >> 3) + (kk & 7) * 2;
        *reinterpret_cast<__half*>(hi + o) = h;
        *reinterpret_cast<__half*>(lo + o) = __float2half_rn(v - __half2float(h));
    }
    for (int i = threadIdx.x; i < P::FS + P::FST; i += NTHREADS)
        sm.ctab[i] = i < P::FS ? a.chan_sub[i] : a.chan_step[i - P::FS];
    fence_async_smem();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem_base;

    if (warp < W_TW) {
        // ================================================================ producer
        // thread = TMEM lane = A1 row (b, n2) of the pair: b = tp / 64, n2 = tp % 64; its row holds
        // x_hi (n1, re|im) in columns 0-31 and x_lo in 32-63 of the stage
        const int tp = threadIdx.x;
        const int bsel = tp >> 6, n2 = tp & 63;
        const uint32_t lane_off = (uint32_t)(32 * warp) << 16;
        const int npair = nitem * NPAIR;
        for (int g = 0; g < npair; g++) {
            const int x = g % NIB, s = g % NA1;
            const uint32_t ph = (g / NIB) & 1;
            const bool ok = mbar_wait_warp(&sm.cp_full[x], ph, abort_flag) &&
                            mbar_wait_warp(&sm.tab_full[x], ph, abort_flag) &&
                            mbar_wait_warp(&sm.a1_empty[s], ((g / NA1) & 1) ^ 1, abort_flag);
            if (!ok) {   // warp-uniform: the TMEM stores are .sync.aligned
                if (!*abort_flag) atomicCAS(a.err, 0, ERR_WAIT);
                *abort_flag = 1;
                break;
            }
            tc_fence_after();   // the MMAs that read this stage are complete
            const int2 wv = sm.pwin[x][bsel];
            // sample 64 n1 + n2 sits at bit wv.x + 128 n1 + 2 n2 of the staged window: the same shift
            // for every n1, four words apart; two halves of 16 n1 (x_hi columns n1, x_lo 32 + n1)
            const int bit = wv.x + 2 * n2;
            const uint32_t* wp = reinterpret_cast<const uint32_t*>(sm.inb[x][bsel]) + (bit >> 5);
            const int sh = bit & 31;
            const uint2* lt = sm.lut[x][bsel][0];
#pragma unroll
            for (int hf = 0; hf < 2; hf++) {
                uint32_t hv[16], lv[16];
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    const int n1 = 16 * hf + k;
                    const uint2 e = wv.y ? lt[4 * n1 + ((wp[4 * n1] >> sh) & 3u)] : make_uint2(0u, 0u);
                    hv[k] = e.x;
                    lv[k] = e.y;
                }
                if (hf == 1) mbar_arrive(&sm.tab_empty[x]);   // this thread's last read of slot x
                tmem_st16(tmem + lane_off + A1_COL + 64 * s + 16 * hf, hv);
                tmem_st16(tmem + lane_off + A1_COL + 64 * s + 32 + 16 * hf, lv);
            }
            tmem_wait_st();
            tc_fence_before();
            mbar_arrive(&sm.a1_full[s]);
        }
    } else if (warp < W_OUT) {
        // ================================================================ twiddle
        // warp t: lane quarter q = t % 4 (D1 rows 32 q .. 32 q + 31: FFT bsel = q / 2 of the pair,
        // n2 = 32 (q % 2) + lane), pairs h and h + 2 of each item (h = t / 4)
        const int t = warp - W_TW;
        const int q = t & 3, h = t >> 2;
        const int bsel = q >> 1, n2 = 32 * (q & 1) + lane;
        const uint32_t lane_off = (uint32_t)(32 * q) << 16;
        const int khalf = n2 >> 5;
        const uint32_t col = (uint32_t)(((n2 & 31) >> 2) << 4) + 4 * (n2 & 3);   // byte of (n2, re|im) in a row
        const float alpha_n2 = -6.283185307179586f * (float)n2 / (float)F;
        // entries and subband LO of the next item, loaded one item ahead
        DelayEntry dn[2];
        double lon = 0.0;
        if (nitem > 0) {
            for (int u = 0; u < 2; u++) dn[u] = item_entry<TB>(a, 0, ntb, 2 * (h + 2 * u) + bsel);
            lon = a.sb_lo[item_of<TB>(blockIdx.x, a.nant, ntb).sb];
        }
        bool ok = true;
        for (int i = 0; i < nitem && ok; i++) {
            // per pair: start of the twiddle row at k1 = 0 and k1 = 16, and its step e^{i alpha}
            float2 st0[2], st16[2], rho[2];
            {
                const double lo = lon;
                const double lofrac = lo - trunc(lo);
                const bool fraclo = lofrac > 1e-11;   // kernel.c:39
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const DelayEntry d = dn[u];
                    if (d.valid) {
                        // sub[n2]: phase lo (a n2 / F + b') (+ lofrac (int)b), kernel.c:434-470
                        const double intdelay = trunc(d.b);
                        double v = lo * (d.b - intdelay);
                        if (fraclo) v = fma(lofrac, intdelay, v);
                        const double ph = fma((double)n2, lo * d.a * (1.0 / F), v);
                        const float2 sub = cis_half_turns_acc((float)(-2.0 * (ph - trunc(ph))));
                        // alpha: -2 pi n2 / F plus the fractional-sample phase per channel
                        const float al = alpha_n2 + __fmul_rn(sm.ctab[1], __double2float_rn(d.frac));
                        const float2 r = cis_small(al);
                        float2 r16 = cmul(r, r);
                        r16 = cmul(r16, r16);
                        r16 = cmul(r16, r16);
                        r16 = cmul(r16, r16);
                        st0[u] = sub;
                        st16[u] = cmul(sub, r16);
                        rho[u] = r;
                    } else {
                        st0[u] = st16[u] = rho[u] = make_float2(0.f, 0.f);
                    }
                }
            }
            // fstep[k2] (kernel.c:512-523, the step part of the fractional-sample rotator) of FFT
            // 2 h + bsel + 4 (t % 2) of the item, k2 = lane: warp t covers FFT t's row of the table
            {
                const int u = t & 1;
                if (!mbar_wait_warp(&sm.fs_empty[i & 1], ((i >> 1) & 1) ^ 1, abort_flag)) {
                    ok = false;
                    break;
                }
                const DelayEntry d = u ? dn[1] : dn[0];
                float sn = 0.f, cs = 0.f;
                if (d.valid) sincosf(__fmul_rn(sm.ctab[P::FS + lane], __double2float_rn(d.frac)), &sn, &cs);
                sm.fstep[i & 1][lane][2 * (h + 2 * u) + bsel] = make_float2(cs, sn);
                mbar_arrive(&sm.fs_full[i & 1]);
            }
            if (i + 1 < nitem) {
                for (int u = 0; u < 2; u++) dn[u] = item_entry<TB>(a, i + 1, ntb, 2 * (h + 2 * u) + bsel);
                lon = a.sb_lo[item_of<TB>(blockIdx.x + (i + 1) * gridDim.x, a.nant, ntb).sb];
            }
#pragma unroll 1
            for (int j = 0; j < 2 && ok; j++) {
                // tile j = k1 in [16 j, 16 j + 16) of every FFT of the item
                if (!mbar_wait_warp(&sm.a2_empty[j], (i & 1) ^ 1, abort_flag)) {
                    ok = false;
                    break;
                }
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const int p = h + 2 * u;
                    if (j == 0 && !mbar_wait_warp(&sm.d1_full[p], i & 1, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    uint32_t v[32];
                    tmem_ld32(tmem + lane_off + D1_COL + 64 * p + 32 * j, v);
                    tmem_wait_ld();
                    if (j == 1) {
                        tc_fence_before();
                        mbar_arrive(&sm.d1_empty[p]);
                    }
                    const int b = 2 * p + bsel;
                    float2 cur = j ? st16[u] : st0[u];
                    const float2 r = rho[u];
                    // row R = 8 kk + b: R % 8 = b, so the swizzled byte is kk * 1024 + base
                    const uint32_t base = (uint32_t)(b * 128) + (col ^ (uint32_t)(b << 4));
                    uint8_t* hi = sm.a2[j][0][khalf] + base;
                    uint8_t* lo = sm.a2[j][1][khalf] + base;
#pragma unroll
                    for (int kk = 0; kk < 16; kk++) {
                        const float2 y = make_float2(__uint_as_float(v[2 * kk]), __uint_as_float(v[2 * kk + 1]));
                        const float2 z = cmul(y, cur);
                        cur = cmul(cur, r);
                        const uint2 zz = split_pair_t(z.x, z.y);
                        *reinterpret_cast<uint32_t*>(hi + kk * 1024) = zz.x;
                        *reinterpret_cast<uint32_t*>(lo + kk * 1024) = zz.y;
                    }
                }
                if (!ok) break;
                fence_async_smem();
                mbar_arrive(&sm.a2_full[j]);
            }
        }
        if (!ok) {
            if (!*abort_flag) atomicCAS(a.err, 0, ERR_WAIT);
            *abort_flag = 1;
        }
    } else if (warp < W_MMA) {
        // ================================================================ output
        // Two groups of four warps (one per TMEM lane quarter): group g takes half g of every D2
        // tile, channels k2 = 16 g .. 16 g + 15 (32 columns)
        const int q = warp & 3;
        const int g = (warp - W_OUT) >> 2;
        const int r = 32 * q + lane;                // D2 row: k1 % 16 = r / 8, b = r % 8
        const int kl = r >> 3, b = r & 7;
        const uint32_t lane_off = (uint32_t)(32 * q) << 16;
        const int nsig = a.nant;
        bool ok = true;
        int nbox = 0;   // tensor stores of this warp (FP16 output): buffer nbox & 1 is the next to fill
        // bar_or is reached by all output warps in the same order: a failed wait is agreed on at the
        // top of an item before any warp leaves.
        for (int i = 0; i < nitem; i++) {
            const Item it = item_of<TB>(blockIdx.x + i * gridDim.x, a.nant, ntb);
            if (bar_or(2, 32 * NOUT, !ok || *abort_flag)) break;
            // the item's fstep table (twiddle warps)
            if (!mbar_wait_warp(&sm.fs_full[i & 1], (i >> 1) & 1, abort_flag)) ok = false;
            const float2 (*fst)[TB] = sm.fstep[i & 1];
#pragma unroll 1
            for (int j = 0; j < 2; j++) {
                // on an expired wait the warp still takes every barrier of the item (its data are
                // void, the error is recorded) and all output warps stop together at the next item
                if (!mbar_wait_warp(&sm.d2_full[j], i & 1, abort_flag)) ok = false;
                tc_fence_after();
                const int k1 = 16 * j + kl;
                uint32_t v[32];
                tmem_ld32(tmem + lane_off + D2_COL + 64 * j + 32 * g, v);
                tmem_wait_ld();
                tc_fence_before();
                mbar_arrive(&sm.d2_empty[j]);
                if constexpr (OUT16) {
                    // the warp's quarter of the half tile (4 k1 x 16 k2 channels x re|im x 8 FFTs)
                    // goes out as one tensor store from its double-buffered shared box, once the
                    // store that last read this buffer (two stores ago) has read it
                    if (lane == 0) bulk_wait_read_1();
                    __syncwarp();
                    __half* ot = sm.otile[warp - W_OUT][nbox & 1] + (lane >> 3) * (2 * TB) + b;
#pragma unroll
                    for (int kk = 0; kk < 16; kk++) {
                        const int k2 = 16 * g + kk;
                        const float2 y = cmul(make_float2(__uint_as_float(v[2 * kk]), __uint_as_float(v[2 * kk + 1])),
                                              fst[k2][b]);
                        const __half2 hv = __floats2half2_rn(y.x, y.y);
                        ot[kk * (4 * 2 * TB)] = __low2half(hv);
                        ot[kk * (4 * 2 * TB) + TB] = __high2half(hv);
                        if constexpr (AMAX) {
                            // max(|Re|, |Im|) of the stored values over the item's 8 FFTs: the 8 lanes
                            // b = 0..7 of a channel are consecutive (lane = 8 (kl % 4) + b)
                            const __half2 ah = __habs2(hv);
                            uint32_t m = __float_as_uint(fmaxf(__low2float(ah), __high2float(ah)));
                            m = max(m, __shfl_xor_sync(0xffffffffu, m, 1));
                            m = max(m, __shfl_xor_sync(0xffffffffu, m, 2));
                            m = max(m, __shfl_xor_sync(0xffffffffu, m, 4));
                            if (b == 0 && m) atomicMax(a.amax + ((size_t)it.sb * C + k1 + F1 * k2) * nsig + it.ant, m);
                        }
                    }
                    fence_async_smem();   // these writes, visible to the tensor store
                    __syncwarp();
                    if (lane == 0) {
                        // box origin: FFT tb0, row 2 ant, k1 = 16 j + 4 q, k2 = 16 g of subband sb
                        tma_store_4d(&omap, sm.otile[warp - W_OUT][nbox & 1], it.tb0, 2 * it.ant, 16 * j + 4 * q,
                                     K2H * it.sb + 16 * g);
                        bulk_commit();
                    }
                    nbox++;
                } else {
                    float2* pk = reinterpret_cast<float2*>(a.spec) +
                                 (((size_t)it.sb * nsig + it.ant) * a.T + it.tb0 + b) * C + k1;
#pragma unroll
                    for (int kk = 0; kk < 16; kk++) {
                        const int k2 = 16 * g + kk;
                        pk[F1 * k2] = cmul(make_float2(__uint_as_float(v[2 * kk]), __uint_as_float(v[2 * kk + 1])),
                                           fst[k2][b]);
                    }
                }
            }
            mbar_arrive(&sm.fs_empty[i & 1]);   // done with the item's fstep table
        }
        if constexpr (OUT16) {
            if (lane == 0) bulk_wait_all();   // the stores are complete before the CTA exits
        }
        if (!ok) {
            if (!*abort_flag) atomicCAS(a.err, 0, ERR_WAIT);
            *abort_flag = 1;
        }
    } else if (warp >= W_HELP) {
        // ================================================================ helper
        // For each pair, NIB pairs ahead of the producer: the input copies, the tables
        // level(code) * step[n1] as FP16 pairs (step phase lo n1 stride a / F, kernel.c:434-470,
        // one FP64 multiply from the per-FFT slope) and the window offsets.  Helper warp hs takes
        // the pairs g = hs (mod NHELP).
        const int hs = warp - W_HELP;
        const int npair = nitem * NPAIR;
        DelayEntry dn0, dn1;
        double lon = 0.0;
        const uint8_t* rown = nullptr;
        auto fetch = [&](int g, DelayEntry& d0, DelayEntry& d1, double& lo, const uint8_t*& row) {
            const int i = g / NPAIR, p = g % NPAIR;
            d0 = item_entry<TB>(a, i, ntb, 2 * p);
            d1 = item_entry<TB>(a, i, ntb, 2 * p + 1);
            const Item it = item_of<TB>(blockIdx.x + i * gridDim.x, a.nant, ntb);
            lo = a.sb_lo[it.sb];
            row = a.data + ((size_t)it.sb * a.nant + it.ant) * a.pitch;
        };
        if (hs < npair) fetch(hs, dn0, dn1, lon, rown);
        int issued = -1;
        for (int g = hs; g < npair; g += NHELP) {
            const int x = g % NIB;
            const DelayEntry d0 = dn0, d1 = dn1;
            const double lo = lon;
            const uint8_t* row = rown;
            if (g + NHELP < npair) fetch(g + NHELP, dn0, dn1, lon, rown);
            if (!mbar_wait_warp(&sm.tab_empty[x], ((g / NIB) & 1) ^ 1, abort_flag)) {
                if (!*abort_flag) atomicCAS(a.err, 0, ERR_WAIT);
                *abort_flag = 1;
                break;
            }
            if (lane == 0) {
                issue_pair(&sm.cp_full[x], sm.inb[x][0], sm.inb[x][1], row, d0, d1);
                issued = g;
            }
#pragma unroll
            for (int b = 0; b < 2; b++) {
                const DelayEntry& d = b ? d1 : d0;
                uint4 e0 = make_uint4(0u, 0u, 0u, 0u), e1 = e0;
                if (d.valid) {
                    const double phs = (double)(lane * F1) * (lo * d.a * (1.0 / F));
                    const float2 st = cis_half_turns_acc((float)(-2.0 * (phs - trunc(phs))));
                    uint2 v[4];
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        const float lv = level2bit((uint32_t)c);
                        v[c] = split_pair(lv * st.x, lv * st.y);
                    }
                    e0 = make_uint4(v[0].x, v[0].y, v[1].x, v[1].y);
                    e1 = make_uint4(v[2].x, v[2].y, v[3].x, v[3].y);
                }
                uint4* dst = reinterpret_cast<uint4*>(sm.lut[x][b][lane]);
                dst[0] = e0;
                dst[1] = e1;
                if (lane == b) sm.pwin[x][b] = window_bits(d);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&sm.tab_full[x]);
        }
        // this warp's copies must land before the CTA exits (phases already complete return at once)
        if (lane == 0)
            for (int g = issued; g >= 0 && g > issued - NIB; g -= NHELP)
                if (!mbar_drain(&sm.cp_full[g % NIB], (g / NIB) & 1)) {
                    atomicCAS(a.err, 0, ERR_WAIT);
                    sm.drain_fail = 1;
                }
    } else if (warp == W_MMA) {
        // ================================================================ MMA issuer
        // Issue order: step 1 of item 0, then per item i: step-2 tile 0 of i, step 1 of i + 1, step-2
        // tile 1 of i.  Item i + 1's step-1 pairs reuse the D1 slots that the twiddle warps release
        // while they write tile 1 of item i, so those warps find item i + 1's D1 ready instead of
        // waiting behind a whole step-2 tile.
        // The whole warp runs the issue loop and one elected lane issues each group of MMAs and
        // its commits: the descriptors are then warp-uniform values formed outside the divergent
        // issue, and each MMA costs little more than its own instruction in this one thread (a
        // single lane running the whole loop measured slower).  Descriptors: only their low words
        // differ (the high word holds stride, version and swizzle); every operand sits at a fixed
        // offset from the shared-memory block, and a K step of 16 elements is 32 bytes further,
        // i.e. +2 in the start-address field (shared addresses stay below 2^18: the 14-bit field
        // never carries).
        const uint32_t dsm = (uint32_t)umma_desc(smem_u32(&sm));
        auto dlo = [&](const void* p) -> uint32_t {
            return dsm + (uint32_t)(((const char*)p - (const char*)&sm) >> 4);
        };
        auto step1 = [&](int i) -> bool {
            for (int p = 0; p < NPAIR; p++) {
                const int g = i * NPAIR + p;
                const int s = g % NA1;
                if (!mbar_wait_warp(&sm.a1_full[s], (g / NA1) & 1, abort_flag) ||
                    !mbar_wait_warp(&sm.d1_empty[p], (i & 1) ^ 1, abort_flag))
                    return false;
                tc_fence_after();
                const uint32_t d1 = tmem + D1_COL + 64 * p, xa = tmem + A1_COL + 64 * s;
                const uint32_t bh = dlo(sm.b1[0]), bl = dlo(sm.b1[1]);
                // x_hi . W_hi + x_lo . W_hi + x_hi . W_lo; K = 64 = 4 steps of 16 (8 columns,
                // 32 bytes of a 128-byte swizzled row)
                if (elect_one()) {
                    umma_ts_acc<false>(d1, xa, udesc(bh), kIdesc);
#pragma unroll
                    for (int kk = 1; kk < 4; kk++) umma_ts_acc<true>(d1, xa + 8 * kk, udesc(bh + 2 * kk), kIdesc);
#pragma unroll
                    for (int kk = 0; kk < 4; kk++) umma_ts_acc<true>(d1, xa + 32 + 8 * kk, udesc(bh + 2 * kk), kIdesc);
#pragma unroll
                    for (int kk = 0; kk < 4; kk++) umma_ts_acc<true>(d1, xa + 8 * kk, udesc(bl + 2 * kk), kIdesc);
                    umma_commit(&sm.a1_empty[s]);
                    umma_commit(&sm.d1_full[p]);
                }
                __syncwarp();
            }
            return true;
        };
        auto step2 = [&](int i, int j) -> bool {
            if (!mbar_wait_warp(&sm.a2_full[j], i & 1, abort_flag) ||
                !mbar_wait_warp(&sm.d2_empty[j], (i & 1) ^ 1, abort_flag))
                return false;
            tc_fence_after();
            const uint32_t d2 = tmem + D2_COL + 64 * j;
            const uint32_t ah = dlo(sm.a2[j][0][0]), al = dlo(sm.a2[j][1][0]);
            const uint32_t bh = dlo(sm.b2[0][0]), bl = dlo(sm.b2[1][0]);
            constexpr uint32_t AH = sizeof(sm.a2[0][0][0]) >> 4, BH = sizeof(sm.b2[0][0]) >> 4;   // K halves
            // Z_hi . W_hi + Z_lo . W_hi + Z_hi . W_lo; K = 128 = two 64-element halves
#pragma unroll 1
            for (int t = 0; t < 3; t++) {
                const uint32_t a0 = t == 1 ? al : ah, b0 = t == 2 ? bl : bh;
                if (elect_one()) {
                    umma<false>(d2, udesc(a0), udesc(b0), kIdesc, t > 0 ? 1u : 0u);
#pragma unroll
                    for (int kk = 1; kk < 8; kk++)
                        umma_ss_acc<true>(d2, udesc(a0 + (kk >> 2) * AH + 2 * (kk & 3)),
                                          udesc(b0 + (kk >> 2) * BH + 2 * (kk & 3)), kIdesc);
                    if (t == 2) {
                        umma_commit(&sm.a2_empty[j]);
                        umma_commit(&sm.d2_full[j]);
                    }
                }
                __syncwarp();
            }
            return true;
        };
        bool ok = nitem == 0 || step1(0);
        for (int i = 0; i < nitem && ok; i++)
            ok = step2(i, 0) && (i + 1 >= nitem || step1(i + 1)) && step2(i, 1);
        if (!ok && lane == 0) {
            if (!*abort_flag) atomicCAS(a.err, 0, ERR_WAIT);
            *abort_flag = 1;
        }
        // every MMA issued must have retired before TMEM is freed (the commit comes from the lane
        // that issued them: elect.sync elects the same lowest active lane every time)
        if (elect_one()) {
            umma_commit(&sm.drain);
            if (!mbar_drain(&sm.drain, 0)) {
                atomicCAS(a.err, 0, ERR_WAIT);
                sm.drain_fail = 1;
            }
        }
        __syncwarp();
    }

    __syncthreads();
    // after an expired drain, MMAs may still write TMEM: it stays allocated (code 7 was recorded;
    // the context's later tensor-core launches cannot be trusted and the process should reset)
    if (warp == W_MMA && !sm.drain_fail) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

}  // namespace ftc32

bool ftc32_supported(int nchan, int mode, const FArgs& a)
{
    return nchan == ftc32::C && a.npol == 1 && !a.cpx && (a.amax == nullptr || mode == kSpecF16) &&
           a.T % ftc32::TB == 0 &&
           (a.tspan ? a.tspan : a.T) % ftc32::TB == 0 && a.err != nullptr;
}

cudaError_t launch_ftc32(int mode, const FArgs& a, cudaStream_t st)
{
    using namespace ftc32;
    const size_t sm = sizeof(Smem) + 1024;
    const int tspan = a.tspan ? a.tspan : a.T;
    const long long ntask = (long long)a.nsb * a.nant * (tspan / TB);
    if (ntask <= 0) return cudaSuccess;
    if (ntask > 0x7fffffffLL) return cudaErrorInvalidValue;
    int dev = 0, nsm = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const int grid = (int)(ntask < nsm ? ntask : nsm);
    CUtensorMap omap;
    std::memset(&omap, 0, sizeof(omap));
    if (mode == kSpecF16) {
        // FP16 K-major spectra [sb][k2][k1][row][T] (channel k1 + 32 k2) as a 4-D tensor
        // (T, row, k1, 32 sb + k2); boxes of 8 FFTs x 2 rows x 4 k1 x 16 k2 (one output warp's).  T % 8 == 0 keeps
        // every stride a multiple of 16 bytes, and box origins at FFT tb0 (a multiple of 8) keep
        // the innermost coordinate 16-byte aligned.
        auto enc = tc::tensor_map_encoder();
        if (!enc) return cudaErrorNotSupported;
        const cuuint64_t row_b = (cuuint64_t)a.T * 2;
        const cuuint64_t dims[4] = {(cuuint64_t)a.T, (cuuint64_t)a.rows, (cuuint64_t)F1, (cuuint64_t)K2H * a.nsb};
        const cuuint64_t strides[3] = {row_b, row_b * a.rows, row_b * a.rows * F1};
        const cuuint32_t box[4] = {(cuuint32_t)TB, 2, 4, 16};
        const cuuint32_t estr[4] = {1, 1, 1, 1};
        if (enc(&omap, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 4, a.spec, dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
    }
    if (mode == kSpecF16 && a.amax) {
        static unsigned configured = 0;
        if ((e = set_smem_once(k_ftc32<true, true>, sm, &configured)) != cudaSuccess) return e;
        k_ftc32<true, true><<<grid, NTHREADS, sm, st>>>(a, omap);
    } else if (mode == kSpecF16) {
        static unsigned configured = 0;
        if ((e = set_smem_once(k_ftc32<true, false>, sm, &configured)) != cudaSuccess) return e;
        k_ftc32<true, false><<<grid, NTHREADS, sm, st>>>(a, omap);
    } else {
        static unsigned configured = 0;
        if ((e = set_smem_once(k_ftc32<false, false>, sm, &configured)) != cudaSuccess) return e;
        k_ftc32<false, false><<<grid, NTHREADS, sm, st>>>(a, omap);
    }
    return cudaGetLastError();
}

}  // namespace fx
