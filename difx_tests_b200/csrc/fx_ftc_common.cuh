// fx_ftc_common.cuh -- pieces shared by the two tensor-core F stages for 2048-point FFTs of
// one polarisation of 2-bit real input (fx_ftc.cu: FP16 DFT; fx_ftc32.cu: FP32-grade split
// FP16 DFT): swizzled shared-memory addressing, named-barrier OR, work items of TB consecutive
// FFTs of one (subband, antenna), delay entries, input windows and their bulk copies.
#pragma once

#include "fx_fstage.cuh"
#include "fx_tc.cuh"

namespace fx {
namespace ftcc {

constexpr int F = 2048;
constexpr int INB = 544;   // staged bytes per FFT: the 16-byte aligned window plus read-ahead
static_assert(fstage_inb<2048, 1, false>() + 16 <= INB, "staging buffer holds the window and read-ahead");

// 16-byte chunk c of row r of a K-major SWIZZLE_128B tile
__device__ __forceinline__ uint32_t sw128(int r, int c) { return (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4)); }

// bar.red.or over `n` threads on named barrier `id`: true if any thread passed p
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

// work item `task` = (subband, antenna, block of TB FFT slots), slot blocks fastest
template <int TB>
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

// Delay entry of FFT t of item i of this CTA (all zero for slots without data)
template <int TB>
__device__ __forceinline__ DelayEntry item_entry(const FArgs& a, int i, int ntb, int t)
{
    const Item it = item_of<TB>(blockIdx.x + i * gridDim.x, a.nant, ntb);
    DelayEntry d{};
    if (!entry(a, it.ant, it.tb0 + t, d)) d.valid = 0;
    return d;
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

// Input bytes of the two FFTs of a pair (entries d0, d1 of row `row`) into the two buffers of a
// pair slot, by one thread: one arrive.expect_tx on `bar` for both, then the copies.
__device__ __forceinline__ void issue_pair(uint64_t* bar, uint8_t* dst0, uint8_t* dst1, const uint8_t* row,
                                           const DelayEntry& d0, const DelayEntry& d1)
{
    int base[2] = {0, 0}, nvec[2] = {0, 0};
    if (d0.valid) window(d0, base[0], nvec[0]);
    if (d1.valid) window(d1, base[1], nvec[1]);
    tc::mbar_expect_tx(bar, 16u * (nvec[0] + nvec[1]));
    if (d0.valid) bulk_copy(bar, dst0, row + base[0], 16u * nvec[0]);
    if (d1.valid) bulk_copy(bar, dst1, row + base[1], 16u * nvec[1]);
}

// Bit of sample 0 of an FFT inside its staged window, and whether the FFT carries data
__device__ __forceinline__ int2 window_bits(const DelayEntry& d)
{
    int base = 0, nvec = 0;
    if (d.valid) window(d, base, nvec);
    return make_int2(2 * (d.offset - 4 * base), d.valid);
}

}  // namespace ftcc
}  // namespace fx
