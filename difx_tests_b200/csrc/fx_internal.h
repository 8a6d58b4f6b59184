// fx_internal.h -- layouts and launch arguments shared by the host driver and
// the sm_100a kernels of the FX correlator hot path.
//
// Device memory layout (one process call, per subintegration):
//   packed input   u8   [nsb][nant][pitch]        pitch >= subintbytes + 16, 16-B multiple; 2-bit real
//                                                  (reference bit order) or 8-bit complex: int8 (re, im)
//                                                  per polarisation, polarisations interleaved per sample
//   delay table    DelayEntry [nant][ld]           one entry per (antenna, FFT of the call)
//   valid bits     u32  [nant][ld/32]              bit t = antenna valid for FFT t
//   spectra (F32)  f32x2 [nsb][nsig][T][nchan]     plain X stage input, channel-contiguous
//   spectra (F16)  f16  [nsb][nchan][rows][T]      tensor-core X stage input, K(=time)-major;
//                                                  row 2*sig = Re, 2*sig+1 = Im, rows padded
//   spectra (F8)   e4m3 [nsb][nchan][rows][T]      FP8 form: the F16 spectra times 448/absmax
//   absmax         u32  [nsb*nchan][nsig]          FP8 form: float bits of max(|Re|,|Im|) over
//                                                  the chunk, per signal and channel
//   inverse scale  f32  [nsb*nchan][nsig]          FP8 form: absmax/448 (1 when absmax = 0)
//   accumulators   f32x2 [nsb][npair][nchan]       plain form, pair = upper-triangle (i<=j)
//                  f32x2 [nsb][nchan][npair]       tensor-core form
//   counts         i32  [npair_ant]                antenna pairs (a1<=a2) incl. autos
// sig = ant*npol + pol; npair = nsig*(nsig+1)/2 in row-major upper-triangle order.
#pragma once

#include <cstddef>
#include <cstdint>

#include "../../include/fxcorr.h"

namespace fx {

constexpr float kHiMag = 3.3359f;                        // kernel.c:191
constexpr double kNeg2Pi = -2.0 * 3.14159265358979323846;  // -TWO_PI (vectordefs.h:4)

struct DelayEntry {
    double a;       // delay change across the FFT, seconds (kernel.c:383)
    double b;       // delay at the FFT start, seconds (kernel.c:384)
    double frac;    // fractional-sample delay, seconds (kernel.c:739-751)
    int offset;     // integer sample offset of the FFT in the antenna stream
    int valid;      // 0/1 (kernel.c:752-756)
};

enum SpecMode { kSpecF32 = 0, kSpecF16 = 1 };

// device error word bits beyond the tensor-core X stage's wait-expiry codes (1..5)
constexpr int kWindowMiss = 1 << 4;   // an FFT's input was not inside its input window

// Arguments of the fused F-stage kernel (passed by value).
struct FArgs {
    const uint8_t* data;        // packed input [nsb][nant][pitch]
    size_t pitch;
    const DelayEntry* dtab;     // [nant][ld]
    int ld;                     // leading dimension of dtab (FFTs of the call, padded)
    int t_base;                 // dtab column of the chunk's first FFT
    int nfft;                   // FFTs of the chunk that carry data
    int T;                      // FFT slots in the spectra buffer (>= nfft; extra slots zero)
    int nant, npol, nsb;
    const double* sb_lo;        // [nsb] LO per subband, Hz (device)
    const float* chan_sub;      // [stride]     (f32)(2 pi j bw / nchan)       kernel.c:164
    const float* chan_step;     // [nchan/stride] (f32)(2 pi i stride bw / nchan) kernel.c:165
    void* spec;                 // spectra buffer (layout per SpecMode)
    int rows;                   // F16 layout: rows per channel (>= 2*nsig)
    int tb;                     // FFTs per CTA (8, 16 or 32; 0 = 16), chosen by the plan / autotuner
    unsigned* amax;             // F16 layout, FP8 form: running absmax per (sb*nchan + chan, sig), or null
    int tspan;                  // slots [0, tspan) written (>= nfft, multiple of 64; 0 = T)
    int cpx;                    // input format: 0 = 2-bit real, 1 = 8-bit complex (FFT length nchan)
    int* err;                   // device error word (code 6: an input staging wait expired), or null
    int fkind;                  // F-stage arithmetic (FXC_F_FFT32, FXC_F_TC16 or FXC_F_TC32; 0 = FFT32)
};


struct XArgs {
    const void* spec;
    void* acc;
    int nsig, T, nchan, nsb;
    int rows;
    int alt;     // plain-form tile variant: 0 = default, 1 = alternative (chosen by the plan / autotuner)
    const float* inv_scale;   // FP8 form: [nsb*nchan][nsig] factors applied to each Gram product
    int ntk;                  // slots [0, ntk) of each spectra row consumed (0 = T; multiple of 64 / 128 for FP8)
    // plain form with few channel groups: the slots are cut into tseg segments of tlen FFTs (a
    // multiple of 16), each CTA sums one segment into part [tseg][nsb][pair][chan], and a reduce
    // adds the segments to acc in order (tseg <= 1: no segments, CTAs add to acc directly)
    int tseg, tlen;
    void* part;
};

}  // namespace fx
