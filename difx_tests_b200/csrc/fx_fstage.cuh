// fx_fstage.cu -- fused F stage of the FX correlator for sm_100a.
//
// One CTA owns (subband, antenna, block of TB consecutive FFTs).  Per FFT and
// polarisation it performs, without touching HBM in between:
//   K0 lookup  : integer offset / validity / fractional delay from the delay
//                table (kernel.c:733-756, produced by k_delay_table);
//   unpack     : 2-bit decode of F samples starting at `offset` from bytes
//                staged in shared memory by 128-bit loads (kernel.c:397-426);
//   fringe     : multiply by rot[i*S + j] = sub[j] * step[i], the reference's
//                two-level rotator with FP64 phase arguments (kernel.c:428-497);
//   FFT        : forward, unnormalised, length F = 2*nchan (kernel.c:499-510),
//                Stockham radix-16 passes (Govindaraju et al., SC'08) held in
//                registers with padded shared-memory exchanges;
//   frac       : channel c *= fsub[c % stride] * fstep[c / stride]
//                (kernel.c:512-555), channels [0, nchan) only;
//   store      : plain layout [sb][sig][T][nchan] (f32x2), or the FP16 K-major
//                layout [sb][nchan][rows][T] for the tensor-core X stage.  The
//                reference's conjugation (kernel.c:557-568) is folded into the X
//                stage's arithmetic.
#pragma once

#include <algorithm>
#include <cstdio>

#include "fx_common.cuh"
#include "fx_kernels.h"

namespace fx {

constexpr int ilog2c(int x) { return x <= 1 ? 0 : 1 + ilog2c(x / 2); }

// FFT plan of length F.  CPX: complex input (8-bit complex samples), every bin a
// channel (C = F); otherwise real input, channels below F/2 (C = F/2).  Only the
// channel-side constants (C, STRIDE, S, FS, FST, NROT) depend on CPX.
template <int F, bool CPX = false>
struct FPlan {
    static constexpr int C = CPX ? F : F / 2;
    static constexpr int NT = F / 16;                        // threads per FFT
    static constexpr int STRIDE = 1 << (ilog2c(C) / 2);      // kernel.c:31 generalised
    static constexpr int S = F / STRIDE;                      // substride (kernel.c:36)
    static constexpr int FS = STRIDE;                         // frac "sub" length
    static constexpr int FST = C / STRIDE;                    // frac "step" length
    static constexpr int NROT = S + STRIDE + FS + FST;        // rotator table entries
    static constexpr int NPASS = (F == 256) ? 2 : (F <= 4096 ? 3 : 4);
    static constexpr int LASTR = (F == 256) ? 16 : (F == 512) ? 2 : (F == 1024) ? 4 : (F == 2048) ? 8
                               : (F == 4096) ? 16 : 2;
    static constexpr int NSLOT = (NT >= 256) ? 1 : 256 / NT;
    static constexpr int NTHREADS = NT * NSLOT;
    static constexpr int BUF = F + F / 16;                    // padded exchange buffer (float2)
    static constexpr bool TWREG = (F <= 2048);                // twiddles cached in registers
    // pass twiddle tables in shared memory (F > 2048): W256^(r j) [r][j] for pass 1, W4096^(r l) [r][l]
    // and W4096^(16 r h) [r][h] for pass 2 (j = 16 h + l), and for 8192 points W8192^(64 h) [h], W8192^l
    // [l] for pass 3 (j = 64 h + l): a warp's twiddle loads are consecutive or broadcast words (reads of
    // one quarter-wave table at the stride r j conflicted 16 ways), and the tables take 6-7 KB instead
    // of the quarter wave's F / 4 entries, which leaves room for the F16 stage
    static constexpr int TWP = 3 * 256 + (F == 8192 ? 128 : 0);
    static constexpr int MINB = (NTHREADS <= 256) ? 2 : 1;    // CTAs per SM the registers must allow
};

// Staged input bytes per FFT slot: the FFT's bytes (2-bit real: F*npol/4 plus the
// read-ahead byte of kernel.c:402-409; 8-bit complex: 2 bytes per sample and
// polarisation) plus up to 15 bytes of 16-byte alignment slack, rounded to 16.
template <int F, int NPOL, bool CPX>
constexpr int fstage_inb()
{
    return ((CPX ? F * NPOL * 2 : F * NPOL / 4 + 1) + 15 + 15) / 16 * 16;
}

template <int F, int PASS>
struct PassInfo {
    static constexpr int R = (PASS == FPlan<F>::NPASS - 1) ? FPlan<F>::LASTR : 16;
    static constexpr int NS = 1 << (4 * PASS);               // 16^PASS
    static constexpr int NB = 16 / R;                         // butterflies per thread
};

__device__ __forceinline__ int padi(int i) { return i + (i >> 4); }

__device__ __forceinline__ float2 twiddle_exact(int m, int n);

// e^{-2 pi i m / F} for 0 <= m < F: the first-quadrant value e^{-2 pi i m'/F} (m' = m mod F/4)
// turned by the quadrant (exact: swaps and negations)
template <int F>
__device__ __forceinline__ float2 twiddle_q(int m)
{
    const int q = m / (F / 4);
    const float2 b = twiddle_exact(m & (F / 4 - 1), F);
    switch (q & 3) {
    case 0: return b;
    case 1: return make_float2(b.y, -b.x);
    case 2: return make_float2(-b.x, -b.y);
    default: return make_float2(-b.y, b.x);
    }
}

__device__ __forceinline__ float2 twiddle_exact(int m, int n)
{
    float s, c;
    sincospif(-2.0f * (float)m / (float)n, &s, &c);
    return make_float2(c, s);
}

// Stage the packed bytes of one FFT into shared memory with 128-bit loads.  The
// window starts at the 16-byte boundary at or below the FFT's first byte and
// covers the F*npol/4 (+1 when the offset is not byte-aligned, kernel.c:402-409)
// bytes the FFT spans; with the alignment slack that is <= F*npol/4 + 16 bytes.
// Returns the window's base byte index in the antenna row.
__device__ __forceinline__ int stage_fft_bytes(const uint8_t* row, int offset, int npol, int F, uint8_t* inb,
                                               int t, int nthr)
{
    const int first_byte = (npol == 2) ? (offset >> 1) : (offset >> 2);
    const int base_byte = first_byte & ~15;
    const int nvec = (F * npol / 4 + 1 + (first_byte - base_byte) + 15) >> 4;
    const uint4* src = reinterpret_cast<const uint4*>(row + base_byte);
    uint4* dst = reinterpret_cast<uint4*>(inb);
    for (int i = t; i < nvec; i += nthr) dst[i] = __ldg(src + i);
    return base_byte;
}

// Quantiser level of absolute sample s, polarisation pol (kernel.c:397-426 bit
// order for npol=2; 4 consecutive samples per byte, LSB first, for npol=1).
__device__ __forceinline__ float decode_sample(const uint8_t* inb, int base_byte, int s, int npol, int pol)
{
    uint32_t code;
    if (npol == 2) {
        const uint32_t byte = inb[(s >> 1) - base_byte];
        code = (byte >> (4 * (s & 1) + 2 * pol)) & 3u;
    } else {
        const uint32_t byte = inb[(s >> 2) - base_byte];
        code = (byte >> (2 * (s & 3))) & 3u;
    }
    return level2bit(code);
}

template <int NT>
__device__ __forceinline__ void slot_sync(int slot)
{
    if constexpr (NT >= 32) {
        asm volatile("bar.sync %0, %1;" ::"r"(slot + 1), "r"(NT) : "memory");
    } else {
        __syncwarp();
    }
}

// ---- input staging by the bulk-copy (TMA) engine: one cp.async.bulk per FFT into the
// slot's staging buffer, completing an mbarrier phase; every wait is bounded by time.
__device__ __forceinline__ uint32_t smem_u32a(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void stg_bar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32a(bar)) : "memory");
}

// Copy `bytes` (16-byte multiple, both addresses 16-byte aligned) from global src to shared dst.
// The issuing thread orders the slot's earlier reads of dst (made visible to it by a barrier)
// before the async-proxy write.
__device__ __forceinline__ void stg_issue(uint64_t* bar, void* dst, const void* src, uint32_t bytes)
{
    size_t gsrc;
    asm volatile("cvta.to.global.u64 %0, %1;" : "=l"(gsrc) : "l"(src));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32a(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32a(dst)), "l"(gsrc), "r"(bytes), "r"(smem_u32a(bar))
                 : "memory");
}

__device__ __forceinline__ bool stg_try(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32a(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// true when the phase completed, false after 1 s
__device__ __forceinline__ bool stg_wait(uint64_t* bar, uint32_t parity)
{
    if (stg_try(bar, parity)) return true;
    const unsigned long long t0 = gtimer();
    while (!stg_try(bar, parity))
        if (gtimer() - t0 > 1000000000ull) return false;
    return true;
}

// Twiddles a thread needs for pass PASS (r = 0..R-1 of each of its NB butterflies).
template <int F, int PASS>
struct PassTw {
    float2 w[PassInfo<F, PASS>::NB * PassInfo<F, PASS>::R];
};

template <int F, int PASS>
__device__ __forceinline__ void init_pass_tw(PassTw<F, PASS>& tw, int t)
{
    using PI = PassInfo<F, PASS>;
#pragma unroll
    for (int b = 0; b < PI::NB; b++) {
        const int j = t + b * FPlan<F>::NT;
        const int jm = j & (PI::NS - 1);
#pragma unroll
        for (int r = 0; r < PI::R; r++) tw.w[b * PI::R + r] = twiddle_exact(r * jm, PI::NS * PI::R);
    }
}

// Load pass inputs from the exchange buffer and apply the DIT twiddles.  All
// offsets are multiples of 16 elements, so padi(t + c) = padi(t) + c + c/16 and
// every shared-memory access is one base register plus an immediate.
template <int F, int PASS>
__device__ __forceinline__ void pass_load(const float2* buf, const float2* tp, const PassTw<F, PASS>* tw,
                                          float2* v, int t)
{
    using PI = PassInfo<F, PASS>;
    constexpr int NT = FPlan<F>::NT;
    constexpr int STEP = F / PI::R;
    static_assert(STEP % 16 == 0 && NT % 16 == 0, "padded offsets must fold");
    const float2* p0 = buf + padi(t);
#pragma unroll
    for (int b = 0; b < PI::NB; b++) {
        const int jm = (t + b * NT) & (PI::NS - 1);
        const float2* p = p0 + b * (NT + NT / 16);
#pragma unroll
        for (int r = 0; r < PI::R; r++) {
            float2 x = p[r * (STEP + STEP / 16)];
            if (r > 0) {
                float2 w;
                if constexpr (FPlan<F>::TWREG) w = tw->w[b * PI::R + r];
                else if constexpr (PI::NS == 16 && PI::R == 16) w = tp[16 * r + jm];
                else if constexpr (PI::NS == 256 && PI::R == 16)
                    w = cmul(tp[512 + 16 * r + (jm >> 4)], tp[256 + 16 * r + (jm & 15)]);
                else {
                    static_assert(PI::NS == 4096 && PI::R == 2, "every pass of F > 2048 has its table");
                    w = cmul(tp[768 + (jm >> 6)], tp[832 + (jm & 63)]);
                }
                x = cmul(x, w);
            }
            v[b * PI::R + r] = x;
        }
    }
}

template <int F, int PASS>
__device__ __forceinline__ void pass_dft(float2* v)
{
    using PI = PassInfo<F, PASS>;
#pragma unroll
    for (int b = 0; b < PI::NB; b++) dft<PI::R>(v + b * PI::R);
}

// Stockham store: element r of butterfly j goes to (j / NS) * NS * R + j % NS + r * NS.
template <int F, int PASS>
__device__ __forceinline__ void pass_store(float2* buf, const float2* v, int t)
{
    using PI = PassInfo<F, PASS>;
    constexpr int NT = FPlan<F>::NT;
#pragma unroll
    for (int b = 0; b < PI::NB; b++) {
        const int j = t + b * NT;
        float2* p;
        constexpr int RS = (PI::NS == 1) ? 1 : PI::NS + PI::NS / 16;   // padded stride of r
        if constexpr (PI::NS == 1) p = buf + 17 * j;                    // padi(16 j)
        else p = buf + padi((j / PI::NS) * PI::NS * PI::R + (j & (PI::NS - 1)));
#pragma unroll
        for (int r = 0; r < PI::R; r++) p[r * RS] = v[b * PI::R + r];
    }
}

// Rotator table of one FFT: [fr_sub S][fr_step STRIDE][fc_sub FS][fc_step FST].
// Entries are (cos, sin)(pi * x) with x in half-turns, which needs no
// large-argument reduction: fringe x = -2 * frac(phase in turns), i.e. the
// reference's argument -2pi*frac(phase) (kernel.c:463-470) divided by pi;
// fractional-sample x = the reference's float32 argument (kernel.c:517-523) / pi.
// Divisions by F are multiplications by the exact power-of-two reciprocal.
constexpr float kInvPiF = 0.318309886183790671538f;

// Rotator argument x (half-turns) of table entry e; the entry is (cos, sin)(pi x).
template <int F, bool CPX>
__device__ __forceinline__ float rot_arg(int e, const DelayEntry& d, double lo, double lofrac, bool fraclo,
                                         const float* ctab)
{
    using P = FPlan<F, CPX>;
    constexpr double kInvF = 1.0 / F;
    if (e < P::S) {
        // kernel.c:434-466: subphase[j] = lo * (j/F * a + b'), b' = b - (int)b
        const double intdelay = trunc(d.b);
        const double bp = dsub(d.b, intdelay);
        const double xoff = dmul((double)e, kInvF);
        double ph = dmul(dadd(dmul(xoff, d.a), bp), lo);
        if (fraclo) ph = dadd(ph, dmul(lofrac, intdelay));
        return __double2float_rn(-2.0 * dsub(ph, trunc(ph)));
    } else if (e < P::S + P::STRIDE) {
        // kernel.c:145, 452, 469: stepphase[i] = lo * (i*stride/F * a)
        const double xoff = dmul((double)((e - P::S) * P::STRIDE), kInvF);
        const double ph = dmul(dmul(xoff, d.a), lo);
        return __double2float_rn(-2.0 * dsub(ph, trunc(ph)));
    } else {
        const float arg = __fmul_rn(ctab[e - P::S - P::STRIDE], __double2float_rn(d.frac));
        return __fmul_rn(arg, kInvPiF);
    }
}

template <int F, bool CPX>
__device__ __forceinline__ float2 rot_entry(int e, const DelayEntry& d, double lo, double lofrac, bool fraclo,
                                            const float* ctab)
{
    float sn, cs;
    sincospif(rot_arg<F, CPX>(e, d, lo, lofrac, fraclo, ctab), &sn, &cs);
    return make_float2(cs, sn);
}

// One (polarisation, channel) row pair of the F16 layout: NR consecutive FFTs from
// the stage (element q at src[q * CS], Re/Im half2) to the Re row at dst and
// the Im row at dst + T; for the FP8 form also the running absmax.
template <int NR, int NPOL, int C, int CS>
__device__ __forceinline__ void flush_row(const FArgs& args, const __half2* src, int sb, int ant, int pol, int k,
                                          __half* dst)
{
    static_assert(NR >= 4 && NR % 4 == 0, "row segments of 8 bytes or more");
    uint32_t rw[NR / 2], iw[NR / 2];
    __half2 mx = __float2half2_rn(0.f);
#pragma unroll
    for (int q = 0; q < NR / 2; q++) {
        const __half2 h0 = src[(2 * q) * CS];
        const __half2 h1 = src[(2 * q + 1) * CS];
        const __half2 r2 = __lows2half2(h0, h1);
        const __half2 i2 = __highs2half2(h0, h1);
        rw[q] = *reinterpret_cast<const uint32_t*>(&r2);
        iw[q] = *reinterpret_cast<const uint32_t*>(&i2);
        mx = __hmax2(mx, __hmax2(__habs2(h0), __habs2(h1)));
    }
    if (args.amax) {
        // FP8 form: running max(|Re|, |Im|) of the F16 values over the chunk; non-negative
        // floats order like their bit patterns
        const float m = fmaxf(__low2float(mx), __high2float(mx));
        if (m > 0.f) atomicMax(args.amax + ((size_t)sb * C + k) * (args.nant * NPOL) + ant * NPOL + pol,
                               __float_as_uint(m));
    }
    if constexpr (NR == 4) {
        *reinterpret_cast<uint2*>(dst) = make_uint2(rw[0], rw[1]);
        *reinterpret_cast<uint2*>(dst + args.T) = make_uint2(iw[0], iw[1]);
    } else {
#pragma unroll
        for (int q = 0; q < NR / 8; q++) {
            reinterpret_cast<uint4*>(dst)[q] = make_uint4(rw[4 * q], rw[4 * q + 1], rw[4 * q + 2], rw[4 * q + 3]);
            reinterpret_cast<uint4*>(dst + args.T)[q] =
                make_uint4(iw[4 * q], iw[4 * q + 1], iw[4 * q + 2], iw[4 * q + 3]);
        }
    }
}

template <int F>
using Tw2Of = PassTw<F, (FPlan<F>::NPASS > 2 ? 2 : 1)>;

// One F-stage block: TB consecutive FFTs x NPOL of antenna `ant`, subband `sb`,
// starting at chunk slot tb0.  Shared by the single-job grid (k_fstage) and the
// persistent multi-job kernel (k_fstage_batch).
// The slots' staging mbarriers: 16 bytes per slot after the channel table.
template <int F, bool CPX>
__device__ __forceinline__ uint64_t* fstage_bars(unsigned char* smem)
{
    using P = FPlan<F, CPX>;
    float2* rtabs = reinterpret_cast<float2*>(smem) + P::NSLOT * P::BUF + (P::TWREG ? 0 : P::TWP);
    return reinterpret_cast<uint64_t*>(reinterpret_cast<float*>(rtabs + 2 * P::NSLOT * P::NROT) + P::FS + P::FST);
}

template <int F, int MODE, int TB, int NPOL, bool CPX>
__device__ __forceinline__ void fstage_block(const FArgs& args, int sb, int ant, int tb0, unsigned char* smem,
                                             const PassTw<F, 1>& tw1, const Tw2Of<F>& tw2, uint32_t& phase)
{
    using P = FPlan<F, CPX>;
    constexpr int NT = P::NT;
    constexpr int C = P::C;
    constexpr int INB = fstage_inb<F, NPOL, CPX>();                    // staged bytes per slot
    float2* bufs = reinterpret_cast<float2*>(smem);                   // [NSLOT][BUF]
    float2* tq = bufs + P::NSLOT * P::BUF;                              // [TWP] pass twiddle tables
    float2* rtabs = tq + (P::TWREG ? 0 : P::TWP);                      // [NSLOT][2][NROT]
    float* ctab = reinterpret_cast<float*>(rtabs + 2 * P::NSLOT * P::NROT);   // [FS + FST] channel freqs
    uint64_t* bars = reinterpret_cast<uint64_t*>(ctab + P::FS + P::FST);    // [NSLOT] (16 B each)
    uint8_t* inbs = reinterpret_cast<uint8_t*>(bars + 2 * P::NSLOT);        // [NSLOT][INB]
    // [NPOL][TB][CS]: rows padded by 2 half2, so paired flush lanes 8 FFTs apart read other banks
    constexpr int CS = C + 2;
    __half2* stage = reinterpret_cast<__half2*>(inbs + P::NSLOT * INB);
    // one FFT slot per CTA and two polarisations: the stage holds one polarisation's FFTs and is
    // flushed when they are done (items are polarisation-major), so twice the FFT block fits
    constexpr bool PERPOL = (MODE == kSpecF16) && (P::NSLOT == 1) && (NPOL == 2);

    const int tid = threadIdx.x;
    const int slot = tid / NT;
    const int t = tid - slot * NT;
    float2* buf = bufs + slot * P::BUF;
    // rotator tables alternate between two buffers per slot, so the next FFT's table can be
    // written while this FFT's epilogue still reads its own: no barrier between FFTs
    float2* rtab2 = rtabs + slot * 2 * P::NROT;
    uint8_t* inb = inbs + slot * INB;
    uint64_t* bar = bars + 2 * slot;

    const double lo = args.sb_lo[sb];
    const double lofrac = dsub(lo, trunc(lo));
    const bool fraclo = lofrac > 1e-11;                                  // kernel.c:39

    for (int i = tid; i < P::FS + P::FST; i += P::NTHREADS)
        ctab[i] = i < P::FS ? args.chan_sub[i] : args.chan_step[i - P::FS];
    __syncthreads();

    const uint8_t* row = args.data + ((size_t)sb * args.nant + ant) * args.pitch;
    const int nsig = args.nant * NPOL;
    constexpr int NITEM = TB * NPOL;
    const DelayEntry* dtab = args.dtab + (size_t)ant * args.ld + args.t_base;

    // Input window of an item: 16-byte aligned start, nvec 16-byte vectors (2-bit real:
    // F*NPOL/4 bytes + the read-ahead byte of kernel.c:402-409; 8-bit complex: 2*NPOL bytes
    // per sample), copied into the slot's staging buffer by one bulk copy, issued as soon
    // as the previous item's bytes are decoded so the copy overlaps that item's FFT.
    auto window = [&](const DelayEntry& d, int& base, int& nvec) {
        if constexpr (CPX) {
            const int first = d.offset * 2 * NPOL;
            base = first & ~15;
            nvec = (F * NPOL * 2 + (first - base) + 15) >> 4;
        } else {
            const int first = (NPOL == 2) ? (d.offset >> 1) : (d.offset >> 2);
            base = first & ~15;
            nvec = (F * NPOL / 4 + 1 + (first - base) + 15) >> 4;
        }
    };

    // F16 destination of (polarisation, channel) rows of this block
    auto row_dst = [&](int pol, int k) {
        return reinterpret_cast<__half*>(args.spec) +
               (((size_t)sb * C + k) * args.rows + 2 * (ant * NPOL + pol)) * (size_t)args.T + tb0;
    };
    // Flush of every channel's Re/Im rows of polarisations [p0, p0 + np) from stage rows
    // (pol - sp0) * TB + tl, by all threads of the CTA; 32-byte row segments by lane pairs (lanes
    // l and l + 16 take the first and second 8 FFTs of one channel: 16 whole sectors per store).
    auto flush_pols = [&](int p0, int np, int sp0) {
        if constexpr (TB >= 16) {
            for (int e = tid; e < 2 * np * C; e += P::NTHREADS) {
                const int lane = e & 31;
                const int h = lane >> 4;
                const int idx = (e >> 5) * 16 + (lane & 15);
                const int pol = p0 + idx / C;
                const int k = idx % C;
                for (int hb = 0; hb < TB / 16; hb++) {
                    const int tl0 = hb * 16 + h * 8;
                    flush_row<8, NPOL, C, CS>(args, stage + ((pol - sp0) * TB + tl0) * CS + k, sb, ant, pol, k,
                                              row_dst(pol, k) + tl0);
                }
            }
        } else {
            for (int e = tid; e < np * C; e += P::NTHREADS) {
                const int pol = p0 + e / C;
                const int k = e % C;
                flush_row<TB, NPOL, C, CS>(args, stage + ((pol - sp0) * TB) * CS + k, sb, ant, pol, k,
                                           row_dst(pol, k));
            }
        }
    };

    // Items (polarisation-major: item = pol * TB + FFT) are dealt to the slots in
    // contiguous runs of SEG, so with SEG >= 4 every slot owns whole row segments
    // of the F16 layout and flushes them itself, without a CTA-wide barrier.
    constexpr int SEG = (NITEM >= P::NSLOT) ? NITEM / P::NSLOT : 1;
    const int item_end = min(slot * SEG + SEG, NITEM);

    // the first item's delay entry and input copy
    int item = slot * SEG;
    DelayEntry dn;
    bool vn = false;
    int basen = 0, nvecn = 0;
    bool expired = false;   // a staging wait gave up (recorded in *args.err)
    if (item < item_end && tb0 + item % TB < args.nfft) {
        dn = dtab[tb0 + item % TB];
        vn = dn.valid != 0;
    }
    if (vn) {
        window(dn, basen, nvecn);
        if (t == 0) stg_issue(bar, inb, row + basen, 16u * nvecn);
    }

    for (; item < item_end; item++) {
        const int pol = item / TB;
        const int tl = item - pol * TB;
        const int tc = tb0 + tl;                    // FFT slot within the chunk
        float2* rtab = rtab2 + ((item - slot * SEG) & 1) * P::NROT;
        const DelayEntry d = dn;
        const bool valid = vn;
        const int base_byte = basen;
        if (valid) {
            if (!stg_wait(bar, phase)) {
                if (t == 0 && args.err) atomicCAS(args.err, 0, 6);
                expired = true;
            }
            phase ^= 1;
        }
        // ---- the next item of this slot: delay entry now, its copy after this item's decode
        {
            const int ni = item + 1;
            vn = false;
            if (ni < item_end && tb0 + ni % TB < args.nfft) {
                dn = dtab[tb0 + ni % TB];
                vn = dn.valid != 0;
            }
            if (vn) window(dn, basen, nvecn);
        }
        // ---- rotator tables for this FFT (per slot)
        for (int e = t; e < P::NROT; e += NT)
            rtab[e] = valid ? rot_entry<F, CPX>(e, d, lo, lofrac, fraclo, ctab) : make_float2(0.f, 0.f);
        slot_sync<NT>(slot);

        // ---- pass 0: unpack + fringe rotation + radix-16 (samples n = t + r*NT)
        float2 v[16];
        {
            // an invalid item reads from the start of the staging buffer (in range;
            // its rotator is zero, so the levels do not matter)
            const int s0 = valid ? d.offset + t : t;
            const int b0 = valid ? base_byte : 0;
            const uint8_t* bp;
            int sh = 0;
            if constexpr (CPX) {
                // 8-bit complex: (re, im) int8 pairs, polarisations interleaved per sample
                bp = inb + (s0 * 2 * NPOL + 2 * pol - b0);
            } else if constexpr (NPOL == 2) {
                bp = inb + ((s0 >> 1) - b0);
                sh = 4 * (s0 & 1) + 2 * pol;
            } else {
                bp = inb + ((s0 >> 2) - b0);
                sh = 2 * (s0 & 3);
            }
            const float2* fr_sub = rtab;
            const float2* fr_step = rtab + P::S;
            float2 sub_c = make_float2(0.f, 0.f);
            const float2* stp = fr_step;
            if constexpr (NT % P::S == 0) {
                sub_c = fr_sub[t % P::S];   // j = n % S is the same for all r
                stp = fr_step + t / P::S;
            }
#pragma unroll
            for (int r = 0; r < 16; r++) {
                float2 rot;
                if constexpr (NT % P::S == 0) {
                    rot = cmul(sub_c, stp[r * (NT / P::S)]);
                } else {
                    const int n = t + r * NT;
                    rot = cmul(fr_sub[n % P::S], fr_step[n / P::S]);
                }
                if constexpr (CPX) {
                    const char2 c8 = *reinterpret_cast<const char2*>(bp + r * (NT * 2 * NPOL));
                    v[r] = cmul(make_float2((float)c8.x, (float)c8.y), rot);
                } else {
                    const uint32_t byte = bp[r * (NT * NPOL / 4)];
                    const float lv = level2bit((byte >> sh) & 3u);
                    v[r] = make_float2(lv * rot.x, lv * rot.y);
                }
            }
        }
        dft<16>(v);
        pass_store<F, 0>(buf, v, t);
        slot_sync<NT>(slot);
        // this item's bytes are decoded: the next item's copy overlaps the rest of its FFT
        if (vn && t == 0) stg_issue(bar, inb, row + basen, 16u * nvecn);

        // ---- middle passes
        if constexpr (P::NPASS > 2) {
            pass_load<F, 1>(buf, tq, &tw1, v, t);
            slot_sync<NT>(slot);
            pass_dft<F, 1>(v);
            pass_store<F, 1>(buf, v, t);
            slot_sync<NT>(slot);
        }
        if constexpr (P::NPASS > 3) {
            pass_load<F, 2>(buf, tq, nullptr, v, t);
            slot_sync<NT>(slot);
            pass_dft<F, 2>(v);
            pass_store<F, 2>(buf, v, t);
            slot_sync<NT>(slot);
        }
        // ---- last pass
        constexpr int LP = P::NPASS - 1;
        using LI = PassInfo<F, LP>;
        if constexpr (LP == 1) pass_load<F, 1>(buf, tq, &tw1, v, t);
        else if constexpr (LP == 2) pass_load<F, 2>(buf, tq, &tw2, v, t);
        else pass_load<F, 3>(buf, tq, nullptr, v, t);
        // real input: outputs r < R/2 only (channels below F/2); complex input: every output
        constexpr int NOUT = CPX ? LI::R : LI::R / 2;
#pragma unroll
        for (int b = 0; b < LI::NB; b++) {
            if constexpr (CPX) dft<LI::R>(v + b * LI::R);
            else dft_lo<LI::R>(v + b * LI::R);
        }

        // ---- fractional-sample correction + store of channels k = j + r*F/R < C
        constexpr int KSTEP = F / LI::R;
        static_assert(KSTEP % P::FS == 0, "frac rotator index must fold");
        const float2* fc_sub = rtab + P::S + P::STRIDE;
        const float2* fc_step = fc_sub + P::FS;
        const int sig = ant * NPOL + pol;
#pragma unroll
        for (int b = 0; b < LI::NB; b++) {
            const int j = t + b * NT;
            const float2 fsub = fc_sub[j % P::FS];
            const float2* fst = fc_step + j / P::FS;
#pragma unroll
            for (int r = 0; r < NOUT; r++) {
                const float2 fr = cmul(fsub, fst[r * (KSTEP / P::FS)]);
                const float2 y = cmul(fr, v[b * LI::R + r]);
                if constexpr (MODE == kSpecF32) {
                    float2* out = reinterpret_cast<float2*>(args.spec) +
                                  (((size_t)sb * nsig + sig) * args.T + tc) * C + j;
                    if (tc < args.T) out[r * KSTEP] = y;
                } else {
                    stage[((PERPOL ? 0 : pol) * TB + tl) * CS + j + r * KSTEP] = __floats2half2_rn(y.x, y.y);
                }
            }
        }
        // no barrier here: the next FFT writes the other rotator table before its first barrier,
        // and buf only after it (the staging buffer's copy was issued after this FFT's decode)
        if constexpr (PERPOL) {
            if (tl == TB - 1) {       // this polarisation's FFTs are staged (the CTA is one slot)
                slot_sync<NT>(slot);
                flush_pols(pol, 1, pol);
                slot_sync<NT>(slot);  // the next polarisation reuses the stage
            }
        }
    }
    // after an expired wait the copy may still land: wait for it once more (bounded) so it
    // cannot write into the staging buffer of a later task or an exited CTA
    if (expired) stg_wait(bar, phase ^ 1);

    if constexpr (MODE == kSpecF16 && !PERPOL) {
        if constexpr (TB >= 16) {
            // whole row segments by lane pairs; the CTA's 16 FFTs of a row are all staged only
            // after a CTA-wide barrier
            __syncthreads();
            flush_pols(0, NPOL, 0);
        } else if constexpr (SEG >= 4) {
            // flush of this slot's rows: FFTs [tl0, tl0 + NR) of NPS polarisations, once the
            // slot's stage entries are visible to all its threads
            slot_sync<NT>(slot);
            constexpr int NR = SEG < TB ? SEG : TB;
            constexpr int NPS = SEG / NR;
            const int pol0 = (slot * SEG) / TB;
            const int tl0 = (slot * SEG) % TB;
            for (int e = t; e < NPS * C; e += NT) {
                const int pol = pol0 + e / C;
                const int k = e % C;
                flush_row<NR, NPOL, C, CS>(args, stage + (pol * TB + tl0) * CS + k, sb, ant, pol, k,
                                           row_dst(pol, k) + tl0);
            }
        } else {
            __syncthreads();
            flush_pols(0, NPOL, 0);   // one (pol, channel) per thread, TB FFTs each
        }
    }
}

// Per-CTA set-up shared by both kernels: the quarter-wave twiddle table (large
// F) or the thread's register twiddles (F <= 2048); job independent.
template <int F>
__device__ __forceinline__ void fstage_prologue(unsigned char* smem, PassTw<F, 1>& tw1, Tw2Of<F>& tw2)
{
    using P = FPlan<F>;
    const int tid = threadIdx.x;
    const int t = tid % P::NT;
    if constexpr (!P::TWREG) {
        float2* tp = reinterpret_cast<float2*>(smem) + P::NSLOT * P::BUF;
        for (int e = tid; e < P::TWP; e += P::NTHREADS) {
            int m;
            if (e < 768) {
                const int k = e >> 8, r = (e >> 4) & 15, j = e & 15;
                m = k == 0 ? r * j * (F / 256) : (k == 1 ? r * j : 16 * r * j) * (F / 4096);
            } else {
                m = e < 832 ? 64 * (e - 768) : e - 832;   // 8192 points, pass 3
            }
            tp[e] = twiddle_q<F>(m);
        }
    } else {
        init_pass_tw<F, 1>(tw1, t);
        if constexpr (P::NPASS > 2) init_pass_tw<F, 2>(tw2, t);
    }
}

// One staging mbarrier per FFT slot, initialised by the slot's first thread before the
// block's first barrier (fstage_block's channel-table __syncthreads) orders it before use.
template <int F, bool CPX>
__device__ __forceinline__ void fstage_bars_init(unsigned char* smem)
{
    using P = FPlan<F, CPX>;
    if (threadIdx.x % P::NT == 0) {
        stg_bar_init(fstage_bars<F, CPX>(smem) + 2 * (threadIdx.x / P::NT));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
}

// Single job: grid (T / TB, nant, nsb).
template <int F, int MODE, int TB, int NPOL, bool CPX>
__global__ void __launch_bounds__(FPlan<F>::NTHREADS, FPlan<F>::MINB)
k_fstage(FArgs args)
{
    extern __shared__ __align__(16) unsigned char smem[];
    PassTw<F, 1> tw1;
    Tw2Of<F> tw2;
    fstage_prologue<F>(smem, tw1, tw2);
    fstage_bars_init<F, CPX>(smem);
    uint32_t phase = 0;
    fstage_block<F, MODE, TB, NPOL, CPX>(args, blockIdx.z, blockIdx.y, blockIdx.x * TB, smem, tw1, tw2, phase);
}

// Many jobs in one persistent launch: CTAs stride over a task table
// {job, subband, antenna, first slot}; every job of the launch has this F, NPOL
// and spectra layout, each its own FArgs (2-bit real input).
template <int F, int MODE, int TB, int NPOL>
__global__ void __launch_bounds__(FPlan<F>::NTHREADS, FPlan<F>::MINB)
k_fstage_batch(const FArgs* __restrict__ jobs, const int4* __restrict__ tasks, int ntask)
{
    extern __shared__ __align__(16) unsigned char smem[];
    PassTw<F, 1> tw1;
    Tw2Of<F> tw2;
    fstage_prologue<F>(smem, tw1, tw2);
    fstage_bars_init<F, false>(smem);
    uint32_t phase = 0;
    for (int i = blockIdx.x; i < ntask; i += gridDim.x) {
        const int4 tk = tasks[i];
        const FArgs a = jobs[tk.x];
        fstage_block<F, MODE, TB, NPOL, false>(a, tk.y, tk.z, tk.w, smem, tw1, tw2, phase);
        __syncthreads();   // the next task rewrites the channel table and staging buffers
    }
}

template <int F, bool CPX = false>
size_t fstage_smem(int mode, int tb, int npol)
{
    using P = FPlan<F, CPX>;
    size_t s = (size_t)P::NSLOT * P::BUF * sizeof(float2);
    if (!P::TWREG) s += (size_t)P::TWP * sizeof(float2);
    s += (size_t)2 * P::NSLOT * P::NROT * sizeof(float2);
    s += (size_t)(P::FS + P::FST) * sizeof(float);
    s += (size_t)P::NSLOT * 16;   // staging mbarriers
    s += (size_t)P::NSLOT * (npol == 2 ? fstage_inb<F, 2, CPX>() : fstage_inb<F, 1, CPX>());
    // F16 stage: [npol][tb][C + 2] half2, one polarisation at a time when the CTA is one slot
    if (mode == kSpecF16) s += (size_t)(P::NSLOT == 1 ? 1 : npol) * tb * (P::C + 2) * sizeof(__half2);
    return s;
}

template <int F, int MODE, int TB, int NPOL, bool CPX>
cudaError_t launch_f(const FArgs& a, cudaStream_t st)
{
    using P = FPlan<F, CPX>;
    const size_t sm = fstage_smem<F, CPX>(MODE, TB, NPOL);
    auto kern = k_fstage<F, MODE, TB, NPOL, CPX>;
    static unsigned configured = 0;  // per instantiation and device
    cudaError_t e = set_smem_once(kern, sm, &configured);
    if (e != cudaSuccess) return e;
    dim3 grid(((a.tspan ? a.tspan : a.T) + TB - 1) / TB, a.nant, a.nsb);
    kern<<<grid, P::NTHREADS, sm, st>>>(a);
    return cudaGetLastError();
}

template <int F, int MODE, int TB, int NPOL>
cudaError_t launch_fb(const FArgs* d_jobs, const int4* d_tasks, int ntask, cudaStream_t st)
{
    using P = FPlan<F>;
    const size_t sm = fstage_smem<F>(MODE, TB, NPOL);
    auto kern = k_fstage_batch<F, MODE, TB, NPOL>;
    static unsigned configured = 0;
    cudaError_t e = set_smem_once(kern, sm, &configured);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, P::NTHREADS, sm)) != cudaSuccess) return e;
    const int grid = std::max(1, std::min(ntask, nsm * std::max(1, per_sm)));
    kern<<<grid, P::NTHREADS, sm, st>>>(d_jobs, d_tasks, ntask);
    return cudaGetLastError();
}

// FFT block size: the plan's (0: 16), reduced while the F16 staging (tb FFTs x npol x nchan)
// does not fit the opt-in shared memory (down to 4: 8-byte row segments).
template <int F, bool CPX>
int fstage_tb(int mode, const FArgs& a)
{
    int tb = a.tb ? a.tb : 16;
    if (CPX && tb > 16) tb = 16;   // complex input: 4, 8 and 16 FFTs per CTA are built
    if (mode == kSpecF16) {
        const size_t lim = smem_optin_limit();
        while (tb > 4 && fstage_smem<F, CPX>(mode, tb, a.npol) > lim) tb /= 2;
        // where the registers allow two CTAs per SM, keep the staging small enough for two
        // (their latency hiding outweighs longer row segments)
        if (FPlan<F>::MINB >= 2) {
            const size_t half = smem_per_sm_limit() / 2 - 1024;   // 1 KB reserved per CTA
            int t2 = tb;
            while (t2 > 4 && fstage_smem<F, CPX>(mode, t2, a.npol) > half) t2 /= 2;
            if (fstage_smem<F, CPX>(mode, t2, a.npol) <= half) tb = t2;
        }
    }
    return tb;
}

// Entry points of one FFT length, instantiated in its own translation unit.
template <int F>
cudaError_t launch_fstage_F(int mode, const FArgs& a, cudaStream_t st)
{
    if constexpr (F <= 4096) if (a.cpx) {   // complex FFT length = nchan <= 4096
        const int tb = fstage_tb<F, true>(mode, a);
#define FX_TBC(TBV)                                                                                          \
    if (tb == TBV) {                                                                                         \
        if (mode == kSpecF32) return a.npol == 2 ? launch_f<F, kSpecF32, TBV, 2, true>(a, st)               \
                                                 : launch_f<F, kSpecF32, TBV, 1, true>(a, st);              \
        return a.npol == 2 ? launch_f<F, kSpecF16, TBV, 2, true>(a, st) : launch_f<F, kSpecF16, TBV, 1, true>(a, st); \
    }
        if (tb == 4 && mode == kSpecF16)
            return a.npol == 2 ? launch_f<F, kSpecF16, 4, 2, true>(a, st) : launch_f<F, kSpecF16, 4, 1, true>(a, st);
        FX_TBC(8)
        FX_TBC(16)
#undef FX_TBC
        return cudaErrorInvalidValue;
    }
    const int tb = fstage_tb<F, false>(mode, a);
    if (tb == 4 && mode == kSpecF16)
        return a.npol == 2 ? launch_f<F, kSpecF16, 4, 2, false>(a, st) : launch_f<F, kSpecF16, 4, 1, false>(a, st);
#define FX_TB(TBV)                                                                                      \
    if (tb == TBV) {                                                                                    \
        if (mode == kSpecF32) return a.npol == 2 ? launch_f<F, kSpecF32, TBV, 2, false>(a, st)         \
                                                 : launch_f<F, kSpecF32, TBV, 1, false>(a, st);        \
        return a.npol == 2 ? launch_f<F, kSpecF16, TBV, 2, false>(a, st)                                \
                           : launch_f<F, kSpecF16, TBV, 1, false>(a, st);                               \
    }
    FX_TB(8)
    FX_TB(16)
    FX_TB(32)
#undef FX_TB
    return cudaErrorInvalidValue;
}

template <int F>
cudaError_t launch_fstage_batch_F(int mode, int npol, int tb, const FArgs* d_jobs, const int4* d_tasks, int ntask,
                                  cudaStream_t st)
{
#define FX_TB(TBV)                                                                                         \
    if (tb == TBV) {                                                                                       \
        if (mode == kSpecF32) return npol == 2 ? launch_fb<F, kSpecF32, TBV, 2>(d_jobs, d_tasks, ntask, st) \
                                               : launch_fb<F, kSpecF32, TBV, 1>(d_jobs, d_tasks, ntask, st); \
        return npol == 2 ? launch_fb<F, kSpecF16, TBV, 2>(d_jobs, d_tasks, ntask, st)                      \
                         : launch_fb<F, kSpecF16, TBV, 1>(d_jobs, d_tasks, ntask, st);                     \
    }
    FX_TB(8)
    FX_TB(16)
    FX_TB(32)
#undef FX_TB
    return cudaErrorInvalidValue;
}

}  // namespace fx
