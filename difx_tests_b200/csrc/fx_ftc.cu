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
//   warps 0-3   producer: decode + fringe rotation, two FFTs per A1 stage (ring of 3); the
//               stage's input bytes arrive by bulk copy one stage ahead
//   warps 4-7   twiddle: D1 (TMEM ring of 4) -> twiddles -> A2 (all 16 FFTs, 128 KB)
//   warps 8-11  output: D2 -> fractional-sample rotator -> F16 spectra rows [chan][row][T]
//               (16 FFTs = one 32-byte sector per row); FP8 form: absmax per (chan, signal)
//   warp 12     MMA issuer (one thread), TMEM owner
// Every wait is bounded (1 s): on expiry the CTA records code 7 in the error word, stops,
// drains what it issued and frees TMEM.
#include "fx_fstage.cuh"
#include "fx_tc.cuh"

namespace fx {
namespace ftc {

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
constexpr int NTHREADS = 416;             // 13 warps
constexpr int INB = 544;                  // staged bytes per FFT: the window plus read-ahead
constexpr int NROT = F2 + F1;             // fringe sub[64] | step[32] per FFT
constexpr uint32_t TMEM_COLS = 512;
constexpr uint32_t D2_COL = ND1 * 64;     // D2: 4 tiles x 64 columns
constexpr int ERR_WAIT = 7;
constexpr uint32_t kIdesc = tc::idesc_f16(128, 64);
static_assert(fstage_inb<2048, 1, false>() + 16 <= INB, "staging buffer holds the window and read-ahead");

struct Smem {
    alignas(1024) uint8_t a2[4][2][128 * 128];   // [k1 / 8][K half][row (k1 % 8) * 16 + b]
    alignas(1024) uint8_t a1[NA1][128 * 128];    // [stage][row b * 64 + n2]
    alignas(1024) uint8_t b1[64 * 128];          // [(k1, re|im)][(n1, re|im)]
    alignas(1024) uint8_t b2[2][64 * 128];       // [K half][(k2, re|im)][(n2 % 32, re|im)]
    alignas(16) uint8_t inb[2][2][INB];         // [pair parity][FFT of the pair]
    float2 rtab[2][2][NROT];                     // [pair parity][FFT of the pair]
    float2 fsub[TB][F1];                         // [b][k1]
    float2 fstep[K2H][TB];                       // [k2][b]
    float2 lut[16];                              // two 2-bit codes -> two levels
    float ctab[P::FS + P::FST];                  // chan_sub | chan_step
    uint64_t a1_full[NA1], a1_empty[NA1], d1_full[ND1], d1_empty[ND1];
    uint64_t a2_full, a2_empty, d2_full, d2_empty, drain;
    uint64_t stg[2];
    uint32_t tmem_base;
    int abort;
};
static_assert(sizeof(Smem) + 1024 <= 232448, "fits the opt-in shared memory of one CTA");

// 16-byte chunk c of row r of a K-major SWIZZLE_128B tile
__device__ __forceinline__ uint32_t sw128(int r, int c) { return (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4)); }

__device__ __forceinline__ bool bar_or(int id, int n, bool p)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred pi, po;\n\t"
        "setp.ne.u32 pi, %1, 0;\n\t"
        "bar.red.or.pred po, %2, %3, pi;\n\t"
        "selp.u32 %0, 1, 0, po;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)p), "r"(id), "r"(n)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ uint32_t h2u(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }

struct Item {
    int sb, ant, tb0;
};

__device__ __forceinline__ Item item_of(int task, int nant, int ntb)
{
    Item it;
    it.tb0 = (task % ntb) * TB;
    const int r = task / ntb;
    it.ant = r % nant;
    it.sb = r / nant;
    return it;
}

// delay entry of FFT slot tc of antenna ant; valid only for FFTs that carry data
__device__ __forceinline__ bool entry(const FArgs& a, int ant, int tc, DelayEntry& d)
{
    if (tc >= a.nfft) return false;
    d = a.dtab[(size_t)ant * a.ld + a.t_base + tc];
    return d.valid != 0;
}

__device__ __forceinline__ void bulk_copy(uint64_t* bar, void* dst, const void* src, uint32_t bytes)
{
    size_t gsrc;
    asm volatile("cvta.to.global.u64 %0, %1;" : "=l"(gsrc) : "l"(src));
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(tc::smem_u32(dst)), "l"(gsrc), "r"(bytes), "r"(tc::smem_u32(bar))
                 : "memory");
}

// Input window of an FFT (2-bit real, one polarisation): 16-byte aligned base byte and vectors
__device__ __forceinline__ void window(const DelayEntry& d, int& base, int& nvec)
{
    const int first = d.offset >> 2;
    base = first & ~15;
    nvec = (F / 4 + 1 + (first - base) + 15) >> 4;
}

// Input bytes of the two FFTs of flat pair g, by one thread: one expect_tx for both, then the copies.
__device__ __forceinline__ void issue_pair(const FArgs& a, Smem& sm, int g, int ntb)
{
    const Item it = item_of(blockIdx.x + (g / NPAIR) * gridDim.x, a.nant, ntb);
    const int p = g % NPAIR;
    const uint8_t* row = a.data + ((size_t)it.sb * a.nant + it.ant) * a.pitch;
    int base[2], nvec[2];
    bool v[2];
    uint32_t total = 0;
    for (int b = 0; b < 2; b++) {
        DelayEntry d;
        v[b] = entry(a, it.ant, it.tb0 + 2 * p + b, d);
        if (v[b]) {
            window(d, base[b], nvec[b]);
            total += 16u * nvec[b];
        }
    }
    uint64_t* bar = &sm.stg[g & 1];
    tc::fence_async_smem();   // earlier reads of the buffer (ordered by the producers' barrier)
    tc::mbar_expect_tx(bar, total);
    for (int b = 0; b < 2; b++)
        if (v[b]) bulk_copy(bar, sm.inb[g & 1][b], row + base[b], 16u * nvec[b]);
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
        mbar_init(&sm.stg[0], 1);
        mbar_init(&sm.stg[1], 1);
        sm.abort = 0;
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
        const int tp = threadIdx.x;
        const int bsel = tp >> 6, t64 = tp & 63, o = t64 & 15, h = t64 >> 4;
        const int npair = nitem * NPAIR;
        int issued = -1;   // last flat pair whose copy was issued
        if (tp == 0 && npair > 0) {
            issue_pair(a, sm, 0, ntb);
            issued = 0;
        }
        bool bad = false;
        for (int g = 0; g < npair; g++) {
            const Item it = item_of(blockIdx.x + (g / NPAIR) * gridDim.x, a.nant, ntb);
            const int p = g % NPAIR;
            const int par = g & 1;
            const double lo = a.sb_lo[it.sb];
            const double lofrac = dsub(lo, trunc(lo));
            const bool fraclo = lofrac > 1e-11;   // kernel.c:39
            // fringe rotator tables of the pair's two FFTs
            for (int e = tp; e < 2 * NROT; e += 128) {
                const int b = e / NROT, idx = e - b * NROT;
                DelayEntry d;
                const bool v = entry(a, it.ant, it.tb0 + 2 * p + b, d);
                sm.rtab[par][b][idx] = v ? rot_entry<F, false>(idx, d, lo, lofrac, fraclo, sm.ctab) : make_float2(0.f, 0.f);
            }
            if (bar_or(1, 128, bad || *abort_flag)) break;
            if (tp == 0 && g + 1 < npair) {
                issue_pair(a, sm, g + 1, ntb);
                issued = g + 1;
            }
            const int s = g % NA1;
            if (!mbar_wait(&sm.stg[par], (g >> 1) & 1, abort_flag) ||
                !mbar_wait(&sm.a1_empty[s], ((g / NA1) & 1) ^ 1, abort_flag)) {
                if (!*abort_flag) atomicCAS(a.err, 0, ERR_WAIT);
                *abort_flag = 1;
                bad = true;
                continue;   // leave at the next barrier, together with the other producers
            }
            // 4 consecutive samples n2 = 4o..4o+3 for 8 values n1 = 8h..8h+7 of FFT bsel
            uint32_t res[4][8];
            DelayEntry d;
            if (entry(a, it.ant, it.tb0 + 2 * p + bsel, d)) {
                int base, nvec;
                window(d, base, nvec);
                const int P0 = 2 * (d.offset + 4 * o - 4 * base);   // bit of sample 4o in the window
                const int w0 = P0 >> 5, sh = P0 & 31;
                const uint32_t* wp = reinterpret_cast<const uint32_t*>(sm.inb[par][bsel]);
                const float2* rt = sm.rtab[par][bsel];
                float2 sub[4], stp[8];
#pragma unroll
                for (int i = 0; i < 4; i++) sub[i] = rt[4 * o + i];
#pragma unroll
                for (int i = 0; i < 8; i++) stp[i] = rt[F2 + 8 * h + i];
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
            uint8_t* st = sm.a1[s];
#pragma unroll
            for (int i2 = 0; i2 < 4; i2++) {
                const int r = bsel * 64 + 4 * o + i2;
#pragma unroll
                for (int jj = 0; jj < 2; jj++)
                    *reinterpret_cast<uint4*>(st + sw128(r, 2 * h + jj)) =
                        make_uint4(res[i2][4 * jj], res[i2][4 * jj + 1], res[i2][4 * jj + 2], res[i2][4 * jj + 3]);
            }
            fence_async_smem();
            mbar_arrive(&sm.a1_full[s]);
        }
        // copies must land before the CTA exits: the last one issued, and the one before it when
        // its wait gave up (waits on phases already complete return at once)
        if (tp == 0)
            for (int x = issued - 1; x <= issued; x++)
                if (x >= 0 && !mbar_drain(&sm.stg[x & 1], (x >> 1) & 1)) atomicCAS(a.err, 0, ERR_WAIT);
    } else if (warp < 8) {
        // ================================================================ twiddle
        const int q = warp & 3;
        const int r = 32 * q + lane;                // D1 row: b % 2 = r / 64, n2 = r % 64
        const int bl = r >> 6, n2 = r & 63;
        const int khalf = n2 >> 5, cl = (n2 & 31) >> 2, wd = n2 & 3;
        float2 tw[F1];
#pragma unroll
        for (int k1 = 0; k1 < F1; k1++) tw[k1] = twiddle_exact(n2 * k1, F);
        bool ok = true;
        for (int i = 0; i < nitem && ok; i++) {
            if (!__all_sync(0xffffffffu, mbar_wait(&sm.a2_empty, (i & 1) ^ 1, abort_flag))) {
                ok = false;
                break;
            }
            for (int p = 0; p < NPAIR; p++) {
                const int g = i * NPAIR + p;
                const int dslot = g % ND1;
                // warp-uniform: the TMEM loads below are .sync.aligned
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
        bool ok = true;
        for (int i = 0; i < nitem; i++) {
            const Item it = item_of(blockIdx.x + i * gridDim.x, a.nant, ntb);
            if (bar_or(2, 128, !ok || *abort_flag)) break;   // the previous item's table reads are done
            const double lo = a.sb_lo[it.sb];
            const double lofrac = dsub(lo, trunc(lo));
            const bool fraclo = lofrac > 1e-11;
            for (int e = to; e < TB * (F1 + K2H); e += 128) {
                const bool isub = e < TB * F1;
                const int e2 = isub ? e : e - TB * F1;
                const int bb = isub ? e2 / F1 : e2 % TB;
                const int kx = isub ? e2 % F1 : e2 / TB;
                DelayEntry d;
                const bool v = entry(a, it.ant, it.tb0 + bb, d);
                const int ridx = F2 + F1 + (isub ? kx : P::FS + kx);
                const float2 w = v ? rot_entry<F, false>(ridx, d, lo, lofrac, fraclo, sm.ctab) : make_float2(0.f, 0.f);
                if (isub) sm.fsub[bb][kx] = w;
                else sm.fstep[kx][bb] = w;
            }
            if (bar_or(2, 128, !ok || *abort_flag)) break;
            // warp-uniform (the TMEM loads are .sync.aligned); a thread that gave up leaves at the
            // next barrier together with the rest of the group
            if (!__all_sync(0xffffffffu, mbar_wait(&sm.d2_full, i & 1, abort_flag))) {
                ok = false;
                continue;
            }
            tc_fence_after();
            __half* dst0 = spec + ((size_t)it.sb * C) * chan_stride + (size_t)(2 * it.ant) * a.T + it.tb0 + b;
#pragma unroll 1
            for (int j = 0; j < 4; j++) {
                const int k1 = 8 * j + kl;
                const float2 fs = sm.fsub[b][k1];
#pragma unroll
                for (int hf = 0; hf < 2; hf++) {
                    uint32_t v[32];
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
                        const float2 fr = cmul(fs, sm.fstep[k2][b]);
                        const float2 y = cmul(fr, x);
                        const __half2 hv = __floats2half2_rn(y.x, y.y);
                        const int k = k1 + F1 * k2;
                        __half* dst = dst0 + (size_t)k * chan_stride;
                        dst[0] = __low2half(hv);
                        dst[a.T] = __high2half(hv);
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
    } else if (lane == 0) {
        // ================================================================ MMA issuer
        bool ok = true;
        for (int i = 0; i < nitem && ok; i++) {
            for (int p = 0; p < NPAIR; p++) {
                const int g = i * NPAIR + p;
                const int s = g % NA1, dslot = g % ND1;
                if (!mbar_wait(&sm.a1_full[s], (g / NA1) & 1, abort_flag) ||
                    !mbar_wait(&sm.d1_empty[dslot], ((g / ND1) & 1) ^ 1, abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t sa = smem_u32(sm.a1[s]), sb = smem_u32(sm.b1);
#pragma unroll
                for (int kk = 0; kk < 4; kk++)
                    umma<false>(tmem + dslot * 64, umma_desc(sa + kk * 32), umma_desc(sb + kk * 32), kIdesc,
                                kk > 0 ? 1u : 0u);
                umma_commit(&sm.a1_empty[s]);
                umma_commit(&sm.d1_full[dslot]);
            }
            if (!ok) break;
            if (!mbar_wait(&sm.a2_full, i & 1, abort_flag) || !mbar_wait(&sm.d2_empty, (i & 1) ^ 1, abort_flag)) {
                ok = false;
                break;
            }
            tc_fence_after();
#pragma unroll 1
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int kk = 0; kk < 8; kk++)
                    umma<false>(tmem + D2_COL + 64 * j, umma_desc(smem_u32(sm.a2[j][kk >> 2]) + (kk & 3) * 32),
                                umma_desc(smem_u32(sm.b2[kk >> 2]) + (kk & 3) * 32), kIdesc, kk > 0 ? 1u : 0u);
            umma_commit(&sm.a2_empty);
            umma_commit(&sm.d2_full);
        }
        if (!ok) {
            if (!*abort_flag) atomicCAS(a.err, 0, ERR_WAIT);
            *abort_flag = 1;
        }
        // every MMA issued must have retired before TMEM is freed
        umma_commit(&sm.drain);
        if (!mbar_drain(&sm.drain, 0)) atomicCAS(a.err, 0, ERR_WAIT);
    }

    __syncthreads();
    if (warp == 12) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

}  // namespace ftc

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
