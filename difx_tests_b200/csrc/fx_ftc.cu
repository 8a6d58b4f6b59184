// fx_ftc.cu -- tensor-core F stage (tcgen05) for the FP16 / FP8 X forms: FFT length 2048
// (1024 channels), 2-bit real input, one polarisation.
//
// The DFT of length 2048 is split as 32 x 64 along the factorisation the reference's
// rotators already use (kernel.c:31-36, 160-165: stride 32, substride 64).  With sample
// n = 64 n1 + n2 and channel k = k1 + 32 k2,
//   X[k1 + 32 k2] = sum_n2 W64^(n2 k2) W2048^(n2 k1) sum_n1 W32^(n1 k1) x[64 n1 + n2]
// (W_N = e^{-2 pi i / N}), where x[n] = level(n) * (sub[n2] * step[n1]) is the
// fringe-rotated sample (kernel.c:428-497) and the fractional-sample rotator of channel k
// is fsub[k1] * fstep[k2] (kernel.c:512-555).  Both inner sums are tensor-core GEMMs with
// constant FP16 DFT matrices in real form (FP32 accumulation):
//   step 1   D1[(b, n2)][(k1, re|im)] = A1[(b, n2)][(n1, re|im)] . B1^T     M128 N64 K64
//   twiddle  Z = D1 * W2048^(n2 k1) on the CUDA cores (FP32), stored FP16
//   step 2   D2[(k1, b)][(k2, re|im)] = A2[(k1, b)][(n2, re|im)] . B2^T     M128 N64 K128, k2 < 32
// b = the FFT within a work item of 16 consecutive FFTs of one (subband, antenna).
//
// Persistent, warp-specialised CTA (one per SM):
//   warps 0-3   producer: decode + fringe rotation, two FFTs per A1 stage (ring of 3)
//   warps 4-7   twiddle: D1 (TMEM ring of 4) -> twiddles -> A2 (all 16 FFTs, 128 KB)
//   warps 8-11  output: D2 -> fractional-sample rotator -> F16 spectra rows [chan][row][T]
//               (16 FFTs = one 32-byte sector per row); FP8 form: absmax per (chan, signal)
//   warp 12     MMA issuer (one thread), TMEM owner
//   warp 13     helper: up to four pairs ahead of the producer, the input bulk copies, the
//               fringe rotator tables and the window offsets of each pair
// Selected by fxc_config.fstage = FXC_F_TC16 (FP16 DFT matrices and intermediate: not FP32
// accuracy); the FP8 form's absmax lands on the output warps, this kernel's busiest role.
// Every wait is bounded (1 s): on expiry the CTA records code 7 in the error word, stops,
// drains what it issued and frees TMEM.
#include "fx_ftc_common.cuh"

namespace fx {
namespace ftc {

using namespace ftcc;

using P = FPlan<2048>;
constexpr int F = 2048;
constexpr int C = P::C;                   // 1024 channels
constexpr int F1 = P::STRIDE;             // 32: n1, k1
constexpr int F2 = P::S;                  // 64: n2
constexpr int K2H = C / F1;               // 32: k2 of the kept channels
static_assert(F1 == 32 && F2 == 64 && K2H == 32 && P::FS == F1 && P::FST == K2H, "2048-point split");
constexpr int TB = 16;                    // FFTs per work item
constexpr int NPAIR = TB / 2;             // A1 stages per item
constexpr int NA1 = 3;                    // A1 ring
constexpr int ND1 = 4;                    // D1 ring (64 TMEM columns each)
constexpr int NTHREADS = 448;             // 14 warps
constexpr int NIB = 4;                    // pair slots the helper fills ahead of the producer
constexpr int NROT = F2 + F1;             // fringe sub[64] | step[32] per FFT
constexpr uint32_t TMEM_COLS = 512;
constexpr uint32_t D2_COL = ND1 * 64;     // D2: 4 tiles x 64 columns
constexpr int ERR_WAIT = 7;
constexpr uint32_t kIdesc = tc::idesc_f16(128, 64);

struct Smem {
    alignas(1024) uint8_t a2[4][2][128 * 128];   // [k1 / 8][K half][row (k1 % 8) * 16 + b]
    alignas(1024) uint8_t a1[NA1][128 * 128];    // [stage][row b * 64 + n2]
    alignas(1024) uint8_t b1[64 * 128];          // [(k1, re|im)][(n1, re|im)]
    alignas(1024) uint8_t b2[2][64 * 128];       // [K half][(k2, re|im)][(n2 % 32, re|im)]
    alignas(16) uint8_t inb[NIB][2][INB];       // [pair % NIB][FFT of the pair] input bytes
    float2 rtab[NIB][2][NROT];                   // [pair % NIB][FFT of the pair] fringe sub | step
    int2 pwin[NIB][2];                           // [pair % NIB][FFT] (bit of sample 0 in inb, valid)
    DelayEntry oent[2][TB];                      // output: delay entries [item parity][FFT]
    float2 fsub[TB][F1 + 1];                     // output: [b][k1] (padded row)
    float2 fstep[K2H][TB];                       // output: [k2][b]
    float2 lut[16];                              // two 2-bit codes -> two levels
    float ctab[P::FS + P::FST];                  // chan_sub | chan_step
    uint64_t a1_full[NA1], a1_empty[NA1], d1_full[ND1], d1_empty[ND1];
    uint64_t a2_full, a2_empty, d2_full, d2_empty, drain;
    uint64_t cp_full[NIB], tab_full[NIB], tab_empty[NIB];
    uint32_t tmem_base;
    int abort;
    int drain_fail;                              // a drain wait expired: copies or MMAs may be in flight
};
static_assert(sizeof(Smem) + 1024 <= 232448, "fits the opt-in shared memory of one CTA");

// A1 row of sample n2 = 4 o + i2 of FFT b of a pair: the eight n2 quads a quarter-warp stores
// land in eight different rows mod 8, so its 16-byte stores hit eight different bank groups
__device__ __forceinline__ int a1_row(int b, int o, int i2) { return b * 64 + 8 * i2 + (o & 7) + 32 * (o >> 3); }

// (cos, sin)(pi x) by the special-function unit
__device__ __forceinline__ float2 cis_half_turns(float x)
{
    float sn, cs;
    __sincosf(3.14159265358979f * x, &sn, &cs);
    return make_float2(cs, sn);
}

// Fractional-sample rotator entry: e^{i ctab[j] frac} (kernel.c:512-523), j < FS + FST
__device__ __forceinline__ float2 frac_rot(int j, const DelayEntry& d, const float* ctab)
{
    float sn, cs;
    __sincosf(__fmul_rn(ctab[j], __double2float_rn(d.frac)), &sn, &cs);
    return make_float2(cs, sn);
}

template <bool AMAX>
__global__ void __launch_bounds__(NTHREADS, 1) k_ftc(FArgs a)
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

    // ---- set-up: barriers, TMEM, constant DFT matrices, level table, channel table
    if (threadIdx.x == 0) {
        for (int s = 0; s < NA1; s++) {
            mbar_init(&sm.a1_full[s], 128);
            mbar_init(&sm.a1_empty[s], 1);
        }
        for (int s = 0; s < ND1; s++) {
            mbar_init(&sm.d1_full[s], 1);
            mbar_init(&sm.d1_empty[s], 128);
        }
        mbar_init(&sm.a2_full, 128);
        mbar_init(&sm.a2_empty, 1);
        mbar_init(&sm.d2_full, 1);
        mbar_init(&sm.d2_empty, 128);
        mbar_init(&sm.drain, 1);
        for (int s = 0; s < NIB; s++) {
            mbar_init(&sm.cp_full[s], 1);
            mbar_init(&sm.tab_full[s], 1);
            mbar_init(&sm.tab_empty[s], 128);
        }
        sm.abort = 0;
        sm.drain_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 12) tmem_alloc(&sm.tmem_base, TMEM_COLS);
    // B1[(k1, c)][(n1, c')] and B2[(k2, c)][(n2, c')]: real form of W^(n k), e = (Re, Im) of W:
    // (c, c') = (0, 0) Re, (0, 1) -Im, (1, 0) Im, (1, 1) Re
    for (int e = threadIdx.x; e < 64 * 64 * 3; e += NTHREADS) {
        const int m = e / (64 * 64);          // 0: B1, 1-2: B2 K halves
        const int rem = e - m * 64 * 64;
        const int nb = rem >> 6, kk = rem & 63;
        const int c = nb & 1, cp = kk & 1;
        float2 w;
        uint8_t* base;
        if (m == 0) {
            w = twiddle_exact(((kk >> 1) * (nb >> 1)) & (F1 - 1), F1);
            base = sm.b1;
        } else {
            const int n2 = (m - 1) * 32 + (kk >> 1);
            w = twiddle_exact((n2 * (nb >> 1)) & (F2 - 1), F2);
            base = sm.b2[m - 1];
        }
        const float v = c == 0 ? (cp == 0 ? w.x : -w.y) : (cp == 0 ? w.y : w.x);
        *reinterpret_cast<__half*>(base + sw128(nb, kk >> 3) + (kk & 7) * 2) = __float2half_rn(v);
    }
    if (threadIdx.x < 16) sm.lut[threadIdx.x] = make_float2(level2bit(threadIdx.x & 3), level2bit(threadIdx.x >> 2));
    for (int i = threadIdx.x; i < P::FS + P::FST; i += NTHREADS)
        sm.ctab[i] = i < P::FS ? a.chan_sub[i] : a.chan_step[i - P::FS];
    fence_async_smem();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem_base;

    if (warp < 4) {
        // ================================================================ producer
        // pair g's input bytes, rotator tables and window offsets are in slot g % NIB once
        // cp_full and tab_full complete (the helper warp fills them ahead)
        const int tp = threadIdx.x;
        const int bsel = tp >> 6, t64 = tp & 63, o = t64 & 15, h = t64 >> 4;
        const int npair = nitem * NPAIR;
        for (int g = 0; g < npair; g++) {
            const int x = g % NIB, s = g % NA1;
            const uint32_t ph = (g / NIB) & 1;
            if (!mbar_wait(&sm.cp_full[x], ph, abort_flag) || !mbar_wait(&sm.tab_full[x], ph, abort_flag) ||
                !mbar_wait(&sm.a1_empty[s], ((g / NA1) & 1) ^ 1, abort_flag)) {
                if (!*abort_flag) atomicCAS(a.err, 0, ERR_WAIT);
                *abort_flag = 1;
                break;
            }
            // 4 consecutive samples n2 = 4o..4o+3 for 8 values n1 = 8h..8h+7 of FFT bsel
            uint32_t res[4][8];
            const int2 wv = sm.pwin[x][bsel];
            if (wv.y) {
                const int P0 = wv.x + 8 * o;                 // bit of sample 4o in the window
                const int w0 = P0 >> 5, sh = P0 & 31;
                const uint32_t* wp = reinterpret_cast<const uint32_t*>(sm.inb[x][bsel]);
                const float2* rt = sm.rtab[x][bsel];
                float2 sub[4], stp[8];
#pragma unroll
                for (int k = 0; k < 4; k++) sub[k] = rt[4 * o + k];
#pragma unroll
                for (int k = 0; k < 8; k++) stp[k] = rt[F2 + 8 * h + k];
#pragma unroll
                for (int i1 = 0; i1 < 8; i1++) {
                    const int idx = w0 + 4 * (8 * h + i1);   // 128 bits per n1
                    const uint32_t v = __funnelshift_r(wp[idx], wp[idx + 1], sh);
                    const float2 l01 = sm.lut[v & 15];
                    const float2 l23 = sm.lut[(v >> 4) & 15];
                    const float lv[4] = {l01.x, l01.y, l23.x, l23.y};
#pragma unroll
                    for (int i2 = 0; i2 < 4; i2++) {
                        const float2 rot = cmul(sub[i2], stp[i1]);
                        res[i2][i1] = h2u(__floats2half2_rn(lv[i2] * rot.x, lv[i2] * rot.y));
                    }
                }
            } else {
#pragma unroll
                for (int i2 = 0; i2 < 4; i2++)
#pragma unroll
                    for (int i1 = 0; i1 < 8; i1++) res[i2][i1] = 0u;
            }
            mbar_arrive(&sm.tab_empty[x]);   // this thread's last read of slot x
            uint8_t* st = sm.a1[s];
#pragma unroll
            for (int i2 = 0; i2 < 4; i2++) {
                const int r = a1_row(bsel, o, i2);
#pragma unroll
                for (int jj = 0; jj < 2; jj++)
                    *reinterpret_cast<uint4*>(st + sw128(r, 2 * h + jj)) =
                        make_uint4(res[i2][4 * jj], res[i2][4 * jj + 1], res[i2][4 * jj + 2], res[i2][4 * jj + 3]);
            }
            fence_async_smem();
            mbar_arrive(&sm.a1_full[s]);
        }
    } else if (warp < 8) {
        // ================================================================ twiddle
        const int q = warp & 3;
        const int r = 32 * q + lane;                // D1 row = a1_row(b % 2, o, i2), n2 = 4 o + i2
        const int bl = r >> 6, rr = r & 63;
        const int n2 = 4 * ((rr & 7) + 8 * (rr >> 5)) + ((rr >> 3) & 3);
        const int khalf = n2 >> 5, cl = (n2 & 31) >> 2, wd = n2 & 3;
        float2 tw[F1];
#pragma unroll
        for (int k1 = 0; k1 < F1; k1++) tw[k1] = twiddle_exact(n2 * k1, F);
        bool ok = true;
        for (int i = 0; i < nitem && ok; i++) {
            // warp-uniform (the TMEM loads are .sync.aligned)
            if (!__all_sync(0xffffffffu, mbar_wait(&sm.a2_empty, (i & 1) ^ 1, abort_flag))) {
                ok = false;
                break;
            }
            for (int p = 0; p < NPAIR; p++) {
                const int g = i * NPAIR + p;
                const int dslot = g % ND1;
                if (!__all_sync(0xffffffffu, mbar_wait(&sm.d1_full[dslot], (g / ND1) & 1, abort_flag))) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const int b = 2 * p + bl;
#pragma unroll
                for (int hf = 0; hf < 2; hf++) {
                    uint32_t v[32];
                    tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + dslot * 64 + hf * 32, v);
                    tmem_wait_ld();
                    if (hf == 1) {
                        tc_fence_before();
                        mbar_arrive(&sm.d1_empty[dslot]);
                    }
#pragma unroll
                    for (int kk = 0; kk < 16; kk++) {
                        const int k1 = hf * 16 + kk;
                        const float2 y = make_float2(__uint_as_float(v[2 * kk]), __uint_as_float(v[2 * kk + 1]));
                        const float2 z = cmul(y, tw[k1]);
                        const int R = ((k1 & 7) << 4) + b;
                        *reinterpret_cast<__half2*>(sm.a2[k1 >> 3][khalf] + sw128(R, cl) + wd * 4) =
                            __floats2half2_rn(z.x, z.y);
                    }
                }
            }
            if (!ok) break;
            fence_async_smem();
            mbar_arrive(&sm.a2_full);
        }
        if (!ok) {
            if (!*abort_flag) atomicCAS(a.err, 0, ERR_WAIT);
            *abort_flag = 1;
        }
    } else if (warp < 12) {
        // ================================================================ output
        const int q = warp & 3;
        const int r = 32 * q + lane;                // D2 row: k1 % 8 = r / 16, b = r % 16
        const int kl = r >> 4, b = r & 15;
        const int to = threadIdx.x - 256;
        __half* spec = reinterpret_cast<__half*>(a.spec);
        const size_t chan_stride = (size_t)a.rows * a.T;
        const int nsig = a.nant;
        // item i's entries are in oent[i & 1] before the item's first barrier (written after the
        // previous item's second barrier, loaded into registers one item earlier)
        DelayEntry dnext;
        if (to < TB && nitem > 0) sm.oent[0][to] = item_entry<TB>(a, 0, ntb, to);
        if (to < TB && nitem > 1) dnext = item_entry<TB>(a, 1, ntb, to);
        bool ok = true;
        for (int i = 0; i < nitem; i++) {
            const Item it = item_of<TB>(blockIdx.x + i * gridDim.x, a.nant, ntb);
            // item i's entries visible; every thread is done with item i - 1's tables
            if (bar_or(2, 128, !ok || *abort_flag)) break;
#pragma unroll
            for (int e = to; e < TB * K2H; e += 128) {
                const int bb = e % TB, k2 = e / TB;
                const DelayEntry& d = sm.oent[i & 1][bb];
                sm.fstep[k2][bb] = d.valid ? frac_rot(P::FS + k2, d, sm.ctab) : make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int e = to; e < TB * F1; e += 128) {
                const int bb = e / F1, k1 = e % F1;
                const DelayEntry& d = sm.oent[i & 1][bb];
                sm.fsub[bb][k1] = d.valid ? frac_rot(k1, d, sm.ctab) : make_float2(0.f, 0.f);
            }
            if (bar_or(2, 128, !ok || *abort_flag)) break;
            if (i + 1 < nitem) {
                if (to < TB) sm.oent[(i + 1) & 1][to] = dnext;
                if (to < TB && i + 2 < nitem) dnext = item_entry<TB>(a, i + 2, ntb, to);
            }
            if (!__all_sync(0xffffffffu, mbar_wait(&sm.d2_full, i & 1, abort_flag))) {
                ok = false;
                continue;
            }
            tc_fence_after();
            __half* dst0 = spec + ((size_t)it.sb * C) * chan_stride + (size_t)(2 * it.ant) * a.T + it.tb0 + b;
            const size_t kstep = (size_t)F1 * chan_stride;   // channel k -> k + 32
            const size_t tim = (size_t)a.T;                  // Re row -> Im row
#pragma unroll 1
            for (int j = 0; j < 4; j++) {
                const int k1 = 8 * j + kl;
                const float2 fs = sm.fsub[b][k1];
#pragma unroll
                for (int hf = 0; hf < 2; hf++) {
                    uint32_t v[32];
                    __half* pk = dst0 + (size_t)k1 * chan_stride + (size_t)(16 * hf) * kstep;
                    tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + D2_COL + 64 * j + 32 * hf, v);
                    tmem_wait_ld();
                    if (j == 3 && hf == 1) {
                        tc_fence_before();
                        mbar_arrive(&sm.d2_empty);
                    }
#pragma unroll
                    for (int kk = 0; kk < 16; kk++) {
                        const int k2 = 16 * hf + kk;
                        const float2 x = make_float2(__uint_as_float(v[2 * kk]), __uint_as_float(v[2 * kk + 1]));
                        const float2 y = cmul(cmul(fs, sm.fstep[k2][b]), x);
                        const __half2 hv = __floats2half2_rn(y.x, y.y);
                        const int k = k1 + F1 * k2;
                        pk[0] = __low2half(hv);
                        pk[tim] = __high2half(hv);
                        pk += kstep;
                        if constexpr (AMAX) {
                            // max(|Re|, |Im|) over the item's 16 FFTs: lanes 0-15 and 16-31 hold
                            // channels k1 and k1 + 1
                            const __half2 ah = __habs2(hv);
                            const uint32_t m = __float_as_uint(fmaxf(__low2float(ah), __high2float(ah)));
                            const uint32_t mlo = __reduce_max_sync(0xffffffffu, lane < 16 ? m : 0u);
                            const uint32_t mhi = __reduce_max_sync(0xffffffffu, lane < 16 ? 0u : m);
                            if ((lane & 15) == 0) {
                                const uint32_t mm = lane == 0 ? mlo : mhi;
                                if (mm) atomicMax(a.amax + ((size_t)it.sb * C + k) * nsig + it.ant, mm);
                            }
                        }
                    }
                }
            }
        }
        if (!ok) {
            if (!*abort_flag) atomicCAS(a.err, 0, ERR_WAIT);
            *abort_flag = 1;
        }
    } else if (warp == 13) {
        // ================================================================ helper
        // For each pair, NIB pairs ahead of the producer: the input copies, the fringe rotator
        // tables and the window offsets.  The phases are linear in the sample index
        // (kernel.c:434-470): sub[j] has phase lo (j a / F + b') (+ lofrac (int)b when the LO has
        // a fractional part) and step[i] has lo i stride a / F, each evaluated as one FP64
        // multiply-add from per-FFT slope and offset (rounding ~1e-16 of the phase in turns).
        const int npair = nitem * NPAIR;
        DelayEntry dn0, dn1;                 // entries of the next pair
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
        if (npair > 0) fetch(0, dn0, dn1, lon, rown);
        int issued = -1;
        for (int g = 0; g < npair; g++) {
            const int x = g % NIB;
            const DelayEntry d0 = dn0, d1 = dn1;
            const double lo = lon;
            const uint8_t* row = rown;
            if (g + 1 < npair) fetch(g + 1, dn0, dn1, lon, rown);   // in flight during this pair
            if (!__all_sync(0xffffffffu, mbar_wait(&sm.tab_empty[x], ((g / NIB) & 1) ^ 1, abort_flag))) {
                if (!*abort_flag) atomicCAS(a.err, 0, ERR_WAIT);
                *abort_flag = 1;
                break;
            }
            if (lane == 0) {
                issue_pair(&sm.cp_full[x], sm.inb[x][0], sm.inb[x][1], row, d0, d1);
                issued = g;
            }
            const double lofrac = lo - trunc(lo);
            const bool fraclo = lofrac > 1e-11;   // kernel.c:39
#pragma unroll
            for (int b = 0; b < 2; b++) {
                const DelayEntry& d = b ? d1 : d0;
                const double intdelay = trunc(d.b);
                double v = lo * (d.b - intdelay);
                if (fraclo) v = fma(lofrac, intdelay, v);
                const double slope = lo * d.a * (1.0 / F);
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    const int j = lane + 32 * k;
                    const double ph = fma((double)j, slope, v);
                    sm.rtab[x][b][j] = d.valid ? cis_half_turns((float)(-2.0 * (ph - trunc(ph)))) : make_float2(0.f, 0.f);
                }
                const double phs = (double)(lane * F1) * slope;
                sm.rtab[x][b][F2 + lane] = d.valid ? cis_half_turns((float)(-2.0 * (phs - trunc(phs))))
                                                   : make_float2(0.f, 0.f);
                if (lane == b) sm.pwin[x][b] = window_bits(d);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&sm.tab_full[x]);
        }
        // copies must land before the CTA exits (phases already complete return at once)
        if (lane == 0)
            for (int g = issued - (NIB - 1); g <= issued; g++)
                if (g >= 0 && !mbar_drain(&sm.cp_full[g % NIB], (g / NIB) & 1)) {
                    atomicCAS(a.err, 0, ERR_WAIT);
                    sm.drain_fail = 1;
                }
    } else if (warp == 12) {
        // ================================================================ MMA issuer
        // The whole warp runs the issue loop (warp-uniform descriptors) and one elected lane issues
        // each group of MMAs and its commits; a single lane running the loop in a divergent branch
        // spends far longer per MMA (measured on the FP32-grade F stage, fx_ftc32.cu).
        const uint32_t dsm = (uint32_t)umma_desc(smem_u32(&sm));
        auto dlo = [&](const void* p) -> uint32_t {
            return dsm + (uint32_t)(((const char*)p - (const char*)&sm) >> 4);
        };
        constexpr uint32_t AH = sizeof(sm.a2[0][0]) >> 4, BH = sizeof(sm.b2[0]) >> 4;   // K halves
        bool ok = true;
        for (int i = 0; i < nitem && ok; i++) {
            for (int p = 0; p < NPAIR; p++) {
                const int g = i * NPAIR + p;
                const int s = g % NA1, dslot = g % ND1;
                if (!mbar_wait_warp(&sm.a1_full[s], (g / NA1) & 1, abort_flag) ||
                    !mbar_wait_warp(&sm.d1_empty[dslot], ((g / ND1) & 1) ^ 1, abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t da = dlo(sm.a1[s]), db = dlo(sm.b1);
                if (elect_one()) {
                    umma_ss_acc<false>(tmem + dslot * 64, udesc(da), udesc(db), kIdesc);
#pragma unroll
                    for (int kk = 1; kk < 4; kk++)
                        umma_ss_acc<true>(tmem + dslot * 64, udesc(da + 2 * kk), udesc(db + 2 * kk), kIdesc);
                    umma_commit(&sm.a1_empty[s]);
                    umma_commit(&sm.d1_full[dslot]);
                }
                __syncwarp();
            }
            if (!ok) break;
            if (!mbar_wait_warp(&sm.a2_full, i & 1, abort_flag) || !mbar_wait_warp(&sm.d2_empty, (i & 1) ^ 1, abort_flag)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t db = dlo(sm.b2[0]);
#pragma unroll 1
            for (int j = 0; j < 4; j++) {
                const uint32_t da = dlo(sm.a2[j][0]);
                if (elect_one()) {
                    umma_ss_acc<false>(tmem + D2_COL + 64 * j, udesc(da), udesc(db), kIdesc);
#pragma unroll
                    for (int kk = 1; kk < 8; kk++)
                        umma_ss_acc<true>(tmem + D2_COL + 64 * j, udesc(da + (kk >> 2) * AH + 2 * (kk & 3)),
                                          udesc(db + (kk >> 2) * BH + 2 * (kk & 3)), kIdesc);
                    if (j == 3) {
                        umma_commit(&sm.a2_empty);
                        umma_commit(&sm.d2_full);
                    }
                }
                __syncwarp();
            }
        }
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
    if (warp == 12 && !sm.drain_fail) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

}  // namespace ftc

// Failure-path check of the tensor-core kernels' bounded wait: an mbarrier that nothing completes
// (no copy or MMA is ever issued, so nothing is left in flight) runs out after 1 s and records
// code 7, as an expired wait of the tensor-core F stage would.
__global__ void k_expire_wait_tc(int* err)
{
    __shared__ __align__(8) uint64_t bar;
    __shared__ int abort_flag;
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if (!tc::mbar_wait(&bar, 0, &abort_flag)) atomicCAS(err, 0, ftc::ERR_WAIT);
    }
}

cudaError_t launch_expire_wait_tc(int* err, cudaStream_t st)
{
    k_expire_wait_tc<<<1, 32, 0, st>>>(err);
    return cudaGetLastError();
}

bool ftc_supported(int nchan, int mode, const FArgs& a)
{
    return mode == kSpecF16 && nchan == ftc::C && a.npol == 1 && !a.cpx && a.T % ftc::TB == 0 &&
           (a.tspan ? a.tspan : a.T) % ftc::TB == 0 && a.err != nullptr;
}

cudaError_t launch_ftc(const FArgs& a, cudaStream_t st)
{
    using namespace ftc;
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
    if (a.amax) {
        static unsigned configured = 0;
        if ((e = set_smem_once(k_ftc<true>, sm, &configured)) != cudaSuccess) return e;
        k_ftc<true><<<grid, NTHREADS, sm, st>>>(a);
    } else {
        static unsigned configured = 0;
        if ((e = set_smem_once(k_ftc<false>, sm, &configured)) != cudaSuccess) return e;
        k_ftc<false><<<grid, NTHREADS, sm, st>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace fx
