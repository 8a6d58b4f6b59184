// fx_xtc32.cu -- tensor-core X stage on FP32 spectra (tcgen05, FP16 inputs cast in shared
// memory, FP32 accumulation), up to 64 signals.
//
// The same Gram as fx_xtc.cu (per channel G = A A^T over the real-ified, time-major rows
// A[2s] = Re X_s, A[2s+1] = Im X_s; kernel.c:846 with the conjugation of kernel.c:557-568), but
// the operand is read from the plain form's FP32 spectra [sb][sig][T][chan], which the FFT F
// stage writes with channel-contiguous stores.  The FP16 K-major layout the tensor cores need is
// a corner turn (time-contiguous rows); done in the F stage it costs that stage a shared-memory
// stage, barriers and a flush per block of FFTs.  Here it is done on the way into the MMA
// operand: each FP32 value is rounded to FP16 exactly as the F stage would round it
// (round-to-nearest of Re and Im), and the Gram accumulates the same MMAs in the same order, so
// the visibilities are bit-identical to fx_xtc.cu on F16 spectra of the same F stage.
//
// Persistent, warp-specialised CTA per SM; work item = (subband, 4 channels: one 32-byte sector
// of each spectrum row, so every DRAM sector fetched is used once):
//   warp 0     TMA producer: box {4 channels, 32 FFTs, nsig signals} of the FP32 spectra
//              (unswizzled: {Re, Im} of the 4 channels of FFT t of signal s at 1024 s + 32 t)
//              into a ring of FP32 stages (as many as 128 KB holds: 2 at 64 signals, 4 at 32)
//   warp 1     MMA issuer: per stage and channel 2 x tcgen05.mma.kind::f16 M128 N128 K16 on the
//              channel's FP16 tile (A and B descriptors the same tile)
//   warps 2-9  cast: FP32 stage j -> K half j % 2 (FFTs 32 (j % 2) .. + 31) of the four channels'
//              FP16 tiles, 128 rows x 64 FFTs, K-major SWIZZLE_128B, rows >= 2 nsig zero; the two
//              halves of a tile are disjoint, so the cast fills one while the MMAs read the other
//   warps 10-13 epilogue: tcgen05.ld of the four channels' accumulators (512 TMEM columns), Re/Im
//              combination, FP32 accumulate into acc[sb][c][pair(i,j)], i <= j; an item is T / 32
//              stages long, so its epilogue (one accumulator set, not double-buffered) is a small
//              part of it.
// Every wait is bounded by time; on expiry the CTA records an error code, drains what it
// issued (again bounded), frees TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cuda_fp16.h>

#include "fx_common.cuh"
#include "fx_kernels.h"
#include "fx_tc.cuh"

namespace fx {

namespace tcx32 {

constexpr int BT = 32;                       // FFTs per FP32 stage (a K half of the FP16 tiles)
constexpr int CB = 4;                        // channels per work item
constexpr int MAXSIG = 64;
constexpr int RING_BYTES = 2 * MAXSIG * BT * CB * 8;   // 128 KB of FP32 stages ([sig][t][ch] float2):
constexpr int MAXS32 = 8;                    // 2 at 64 signals, 4 at 32, up to 8
constexpr int TILE_BYTES = 128 * 128;        // 128 rows x 64 FP16
constexpr int NCW = 8;                       // cast warps
constexpr int NTHREADS = 32 * (2 + NCW + 4);   // producer, MMA, cast, 4 epilogue warps
constexpr int TMEM_COLS = 512;               // 4 channels x 128 FP32 columns
constexpr uint32_t kIdesc = tc::idesc_f16(128, 128);

struct Smem {
    alignas(1024) uint8_t f32[RING_BYTES];
    alignas(1024) uint8_t f16[CB][TILE_BYTES];
    alignas(8) uint64_t full32[MAXS32];
    uint64_t empty32[MAXS32];
    uint64_t full16[2];                      // per K half
    uint64_t empty16[2];
    uint64_t acc_full;
    uint64_t acc_empty;
    uint64_t drain;
    uint32_t tmem_base;
    int abort;
    int drain_fail;
};

__device__ __forceinline__ void tma_load_4d(const CUtensorMap* map, uint64_t* bar, void* dst, int x, int y, int z,
                                            int w)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
        "[%2];" ::"r"(tc::smem_u32(dst)),
        "l"(map), "r"(tc::smem_u32(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
        : "memory");
}

__device__ __forceinline__ uint32_t pack2(float a, float b)
{
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

}  // namespace tcx32

// err: 0 ok; 1 a stage-full wait expired (cast or MMA); 2 a stage-free wait expired (producer or
//      cast); 3 accumulator wait expired; 4 epilogue wait expired; 5 drain expired
__global__ void __launch_bounds__(tcx32::NTHREADS, 1)
k_xtc32(const __grid_constant__ CUtensorMap tmap, XArgs a, int* err)
{
    using namespace tc;
    using namespace tcx32;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    Smem& sm = *reinterpret_cast<Smem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    volatile int* abort_flag = &sm.abort;

    const int nsig = a.nsig;
    const int npair = nsig * (nsig + 1) / 2;
    const int ncq = a.nchan / CB;                 // channel quads per subband
    const int nitems = a.nsb * ncq;
    const int nk = (a.ntk ? a.ntk : a.T) / BT;    // FP32 stages per item (even)
    const uint32_t stage_bytes = (uint32_t)nsig * BT * CB * 8;
    const int ns32 = min(MAXS32, (int)(RING_BYTES / stage_bytes));   // FP32 stages in flight

    if (threadIdx.x == 0) {
        for (int s = 0; s < ns32; s++) {
            mbar_init(&sm.full32[s], 1);
            mbar_init(&sm.empty32[s], NCW);   // one arrival per cast warp
        }
        for (int h = 0; h < 2; h++) {
            mbar_init(&sm.full16[h], NCW);
            mbar_init(&sm.empty16[h], 1);     // tcgen05.commit of the half's MMAs
        }
        mbar_init(&sm.acc_full, 1);
        mbar_init(&sm.acc_empty, 128);
        mbar_init(&sm.drain, 1);
        sm.abort = 0;
        sm.drain_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // rows 2 nsig .. 127 of every FP16 tile stay zero: the cast writes rows below 2 nsig only
    {
        const int nz = (128 - 2 * nsig) * 8;   // 16-byte chunks per tile
        uint8_t* tiles = &sm.f16[0][0];
        for (int i = threadIdx.x; i < CB * nz; i += NTHREADS) {
            const int tile = i / nz;
            const int rem = i - tile * nz;
            *reinterpret_cast<uint4*>(tiles + (size_t)tile * TILE_BYTES + (2 * nsig + rem / 8) * 128 + (rem % 8) * 16) =
                make_uint4(0u, 0u, 0u, 0u);
        }
        fence_async_smem();
    }
    if (warp == 0) tmem_alloc(&sm.tmem_base, TMEM_COLS);
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem_base;

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            long long issued = 0;
            for (int item = blockIdx.x; item < nitems && !*abort_flag; item += gridDim.x) {
                const int sb = item / ncq;
                const int c0 = (item - sb * ncq) * CB;
                for (int kb = 0; kb < nk; kb++) {
                    if (!mbar_wait(&sm.empty32[stage], phase ^ 1, abort_flag)) {
                        if (!*abort_flag) atomicCAS(err, 0, 2);
                        *abort_flag = 1;
                        break;
                    }
                    mbar_expect_tx(&sm.full32[stage], stage_bytes);
                    tma_load_4d(&tmap, &sm.full32[stage], sm.f32 + (size_t)stage * stage_bytes, c0, kb * BT, 0, sb);
                    issued++;
                    if (++stage == ns32) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
            // drain: the last ns32 fills are the only ones that may still be in flight
            for (int s = 0; s < ns32 && issued > 0; s++) {
                const long long idx = issued - 1 - s;
                if (idx < 0) break;
                const int st = (int)(idx % ns32);
                const uint32_t ph = (uint32_t)((idx / ns32) & 1);
                const unsigned long long t0 = globaltimer();
                while (!mbar_try(&sm.full32[st], ph)) {
                    if (globaltimer() - t0 > WAIT_NS) {
                        atomicCAS(err, 0, 5);
                        sm.drain_fail = 1;
                        break;
                    }
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        const uint32_t dsm = (uint32_t)umma_desc(smem_u32(&sm));
        auto dlo = [&](const void* p) -> uint32_t {
            return dsm + (uint32_t)(((const char*)p - (const char*)&sm) >> 4);
        };
        uint32_t ph16 = 0;   // bit h: phase of K half h
        uint32_t acc_phase = 0;
        for (int item = blockIdx.x; item < nitems && !__any_sync(0xffffffffu, *abort_flag); item += gridDim.x) {
            if (!mbar_wait_warp(&sm.acc_empty, acc_phase ^ 1, abort_flag)) {
                if (lane == 0) {
                    if (!*abort_flag) atomicCAS(err, 0, 3);
                    *abort_flag = 1;
                }
                break;
            }
            tc_fence_after();
            bool ok = true;
            for (int kb = 0; kb < nk; kb++) {
                const int h = kb & 1;
                if (!mbar_wait_warp(&sm.full16[h], (ph16 >> h) & 1, abort_flag)) {
                    if (lane == 0) {
                        if (!*abort_flag) atomicCAS(err, 0, 1);
                        *abort_flag = 1;
                    }
                    ok = false;
                    break;
                }
                tc_fence_after();
                if (elect_one()) {
                    // the Gram of each channel's tile over K half h: K16 steps 2h, 2h + 1 (32 bytes of
                    // K each, +2 in the descriptors' start field)
#pragma unroll
                    for (int c = 0; c < CB; c++) {
                        const uint32_t dt = dlo(sm.f16[c]) + 4 * h;
                        const uint32_t d = tmem + c * 128;
                        umma<false>(d, udesc(dt), udesc(dt), kIdesc, kb > 0 ? 1u : 0u);
                        umma<false>(d, udesc(dt + 2), udesc(dt + 2), kIdesc, 1u);
                    }
                    umma_commit(&sm.empty16[h]);
                }
                __syncwarp();
                ph16 ^= 1u << h;
            }
            if (!ok) break;
            if (elect_one()) umma_commit(&sm.acc_full);
            __syncwarp();
            acc_phase ^= 1;
        }
        // drain: every issued MMA retires before TMEM is freed (committed by the issuing lane)
        if (elect_one()) {
            umma_commit(&sm.drain);
            const unsigned long long t0 = globaltimer();
            while (!mbar_try(&sm.drain, 0)) {
                if (globaltimer() - t0 > WAIT_NS) {
                    atomicCAS(err, 0, 5);
                    sm.drain_fail = 1;
                    break;
                }
            }
        }
        __syncwarp();
    } else if (warp < 2 + NCW) {
        // ------------------------------------------------------------ cast (warps 2 .. 1 + NCW)
        // Lane t takes FFT t of the stage for signals s = warp - 2, + NCW, ...: two 16-byte reads
        // of {Re, Im} of the four channels per (s, t).  The 8 lanes of FFTs 8q .. 8q+7 then
        // transpose through shuffles: lane L writes word L % 4 (FFTs 2w, 2w+1) of the Re (L % 8 < 4)
        // or Im row of signal s, chunk 4h + q, in each channel's tile (the Re and Im rows' chunks
        // differ after the swizzle, so the 8 lanes of a group hit 8 banks; groups q and q ^ 1 meet,
        // so a store takes at most two bank passes).
        const int t = lane;
        const int kq = t >> 3;
        const int w = lane & 3;
        const int part = (lane >> 2) & 1;                  // 0: Re row, 1: Im row
        const int srcA = (lane & ~7) + 2 * w;              // lanes of FFTs 8q + 2w, 8q + 2w + 1
        const uint32_t sel = part ? 0x7632u : 0x5410u;     // high or low halves of (Re, Im) pairs
        int s32 = 0;
        uint32_t ph32 = 0;
        uint32_t ph16 = 0;   // bit h: phase of K half h
        bool stop = false;
        for (int item = blockIdx.x; item < nitems && !stop; item += gridDim.x) {
            for (int kb = 0; kb < nk; kb++) {
                const int h = kb & 1;
                if (!mbar_wait_warp(&sm.full32[s32], ph32, abort_flag)) {
                    if (lane == 0) {
                        if (!*abort_flag) atomicCAS(err, 0, 1);
                        *abort_flag = 1;
                    }
                    stop = true;
                    break;
                }
                if (!mbar_wait_warp(&sm.empty16[h], ((ph16 >> h) & 1) ^ 1, abort_flag)) {
                    if (lane == 0) {
                        if (!*abort_flag) atomicCAS(err, 0, 2);
                        *abort_flag = 1;
                    }
                    stop = true;
                    break;
                }
                const uint8_t* src = sm.f32 + (size_t)s32 * stage_bytes;
                const int k = 4 * h + kq;                      // chunk of the 128-byte tile row
                // four signals per pass, their reads issued together (the chain read -> shuffles ->
                // stores of one signal is latency-bound)
                for (int s0 = warp - 2; s0 < nsig; s0 += 4 * NCW) {
                    float4 v[4][2];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int s = s0 + NCW * u;
                        const float4* p = reinterpret_cast<const float4*>(src + s * 1024 + t * 32);
                        v[u][0] = s < nsig ? p[0] : make_float4(0.f, 0.f, 0.f, 0.f);   // channels c0, c0 + 1
                        v[u][1] = s < nsig ? p[1] : make_float4(0.f, 0.f, 0.f, 0.f);   // channels c0 + 2, c0 + 3
                    }
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int s = s0 + NCW * u;
                        if (s >= nsig) break;   // warp-uniform: s depends on the warp only
                        const uint32_t hc[4] = {pack2(v[u][0].x, v[u][0].y), pack2(v[u][0].z, v[u][0].w),
                                                pack2(v[u][1].x, v[u][1].y), pack2(v[u][1].z, v[u][1].w)};
                        const int row = 2 * s + part;
                        const int off = row * 128 + ((k ^ (row & 7)) << 4) + w * 4;
#pragma unroll
                        for (int c = 0; c < CB; c++) {
                            const uint32_t x0 = __shfl_sync(0xffffffffu, hc[c], srcA);
                            const uint32_t x1 = __shfl_sync(0xffffffffu, hc[c], srcA + 1);
                            *reinterpret_cast<uint32_t*>(sm.f16[c] + off) = __byte_perm(x0, x1, sel);
                        }
                    }
                }
                fence_async_smem();   // the tiles are read by the tensor cores (async proxy)
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&sm.empty32[s32]);
                    mbar_arrive(&sm.full16[h]);
                }
                if (++s32 == ns32) {
                    s32 = 0;
                    ph32 ^= 1;
                }
                ph16 ^= 1u << h;
            }
        }
    } else {
        // ------------------------------------------------------------ epilogue (last 4 warps)
        const int q = warp & 3;                  // TMEM lane quadrant of this warp
        const int r = q * 32 + lane;             // accumulator row
        const bool odd = (r & 1) != 0;
        const int i = r >> 1;                    // signal of this row
        const int pbase = i * nsig - (i * (i - 1)) / 2 - i;   // pair(i, j) = pbase + j
        uint32_t acc_phase = 0;
        float2* acc = reinterpret_cast<float2*>(a.acc);
        for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
            const int sb = item / ncq;
            const int c0 = (item - sb * ncq) * CB;
            if (!mbar_wait(&sm.acc_full, acc_phase, abort_flag)) {
                if (!*abort_flag) atomicCAS(err, 0, 4);
                *abort_flag = 1;
                break;
            }
            tc_fence_after();
            for (int c = 0; c < CB; c++) {
                float* out = reinterpret_cast<float*>(acc + ((size_t)sb * a.nchan + c0 + c) * npair);
                const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + c * 128;
#pragma unroll 1
                for (int cq = 0; cq < 4; cq++) {      // 32 columns = 16 signal pairs j per chunk
                    uint32_t v[32];
                    tmem_ld32(taddr + cq * 32, v);
                    tmem_wait_ld();
                    if (c == CB - 1 && cq == 3) {
                        tc_fence_before();
                        mbar_arrive(&sm.acc_empty);
                    }
#pragma unroll
                    for (int jj = 0; jj < 16; jj++) {
                        const int j = cq * 16 + jj;
                        const float g0 = __uint_as_float(v[2 * jj]);      // G[r][2j]
                        const float g1 = __uint_as_float(v[2 * jj + 1]);  // G[r][2j+1]
                        // even row 2i: (G[2i][2j], G[2i][2j+1]) = (a, b); odd row: (c, d).  Re = a + d,
                        // Im = c - b: each row takes the other's column 2j+1
                        const float other = __shfl_xor_sync(0xffffffffu, g1, 1);
                        const float val = odd ? (g0 - other) : (g0 + other);
                        if (j >= i && j < nsig) atomicAdd(out + 2 * (pbase + j) + (odd ? 1 : 0), val);
                    }
                }
            }
            acc_phase ^= 1;
        }
    }

    __syncthreads();
    // after an expired drain, MMAs may still write TMEM: it stays allocated (code 5 was recorded;
    // the context's later tensor-core launches cannot be trusted and the process should reset)
    if (warp == 0 && !sm.drain_fail) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

static size_t xtc32_smem() { return sizeof(tcx32::Smem) + 1024; }

cudaError_t launch_xtc32(const XArgs& a, int* d_err, int nsm, cudaStream_t st)
{
    using namespace tcx32;
    const int nslot = a.ntk ? a.ntk : a.T;
    if (a.nsig < 1 || a.nsig > MAXSIG || a.nchan < CB || a.nchan % CB != 0 || a.T % BT != 0 || nslot % (2 * BT) != 0 ||
        nslot > a.T || a.nsb < 1 || !a.spec || !a.acc)
        return cudaErrorInvalidValue;
    if (xtc32_smem() > 227 * 1024) return cudaErrorInvalidValue;
    auto enc = tc::tensor_map_encoder();
    if (!enc) return cudaErrorNotSupported;
    // FP32 spectra [sb][sig][T][chan] (8-byte complex elements): box {4 channels, 32 FFTs, nsig, 1},
    // unswizzled (dense 16-byte rows: with a swizzle, rows narrower than the swizzle span are each
    // padded to a whole 128-byte line)
    CUtensorMap map;
    const cuuint64_t dims[4] = {(cuuint64_t)a.nchan, (cuuint64_t)a.T, (cuuint64_t)a.nsig, (cuuint64_t)a.nsb};
    const cuuint64_t strides[3] = {(cuuint64_t)a.nchan * 8, (cuuint64_t)a.T * a.nchan * 8,
                                   (cuuint64_t)a.nsig * a.T * a.nchan * 8};
    const cuuint32_t box[4] = {(cuuint32_t)CB, (cuuint32_t)BT, (cuuint32_t)a.nsig, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_INT64, 4, const_cast<void*>(a.spec), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    const size_t sm = xtc32_smem();
    static unsigned configured = 0;
    cudaError_t e = set_smem_once(k_xtc32, sm, &configured);
    if (e != cudaSuccess) return e;
    const long long nitems = (long long)a.nsb * (a.nchan / CB);
    const int grid = nitems < nsm ? (int)nitems : nsm;
    k_xtc32<<<grid, NTHREADS, sm, st>>>(map, a, d_err);
    return cudaGetLastError();
}

}  // namespace fx
