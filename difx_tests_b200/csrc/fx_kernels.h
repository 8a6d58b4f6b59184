// fx_kernels.h -- host-side launchers of the sm_100a kernels (internal).
#pragma once

#include <cuda_runtime.h>

#include "fx_internal.h"

namespace fx {

cudaError_t launch_delay_table(const double* delays, const double* fileoffsets, const int* fftindex, int first,
                               int nant, int nfft, int ld, int F, int maxoffset, double sampletime, DelayEntry* tab,
                               uint32_t* vbits, cudaStream_t st);
// as launch_delay_table, for input windows: antenna a's rows start at sample win[a] and hold
// win[nant + a] samples (device doubles holding integers; spb samples per byte); FFTs not inside
// their window are left out and set kWindowMiss in *err
cudaError_t launch_delay_table_window(const double* delays, const double* fileoffsets, const int* fftindex,
                                      int first, int nant, int nfft, int ld, int F, int maxoffset, double sampletime,
                                      const double* win, int spb, int* err, DelayEntry* tab, uint32_t* vbits,
                                      cudaStream_t st);
cudaError_t launch_counts(const uint32_t* vbits, int nant, int nwords, int* counts, cudaStream_t st);
cudaError_t launch_finalize(const float2* acc, int acc_layout, int nsig, int npol, int nant, int nchan, int nsb,
                            const int* counts, int normalize, float2* vis, cudaStream_t st);
cudaError_t launch_amp_phase(float2* vis, long long n, cudaStream_t st);
cudaError_t launch_fstage(int nchan, int mode, const FArgs& a, cudaStream_t st);
// tensor-core F stage (F16 layout, 2048-point FFTs of one polarisation of 2-bit real input)
bool ftc_supported(int nchan, int mode, const FArgs& a);
cudaError_t launch_ftc(const FArgs& a, cudaStream_t st);
// FP32-grade tensor-core F stage (error-compensated FP16 pairs), same geometry, F16 or F32 layout
bool ftc32_supported(int nchan, int mode, const FArgs& a);
cudaError_t launch_ftc32(int mode, const FArgs& a, cudaStream_t st);
size_t fstage_smem_bytes(int nchan, int mode, int npol, int tb);
cudaError_t launch_fstage_batch(int nchan, int npol, int mode, int tb, const FArgs* d_jobs, const int4* d_tasks,
                                int ntask, cudaStream_t st);
cudaError_t launch_xplain_reduce(const XArgs& a, cudaStream_t st);
void xplain_segments(int nsig, int nchan, int nsb, int T, int nsm, int* tseg, int* tlen);
void xplain_segment_model(long long ctas, long long slots, int T, int* tseg, int* tlen);
int xplain_segments_used(const XArgs& a);
cudaError_t launch_xplain(const XArgs& a, cudaStream_t st);
cudaError_t launch_xplain_batch(int nsig, int alt, const XArgs* d_jobs, const int4* d_tasks, int ntask,
                                cudaStream_t st);
int xplain_channel_group(int nsig, int alt);
cudaError_t launch_xtc(const XArgs& a, int* d_err, int nsm, cudaStream_t st);
// the same Gram on the plain form's FP32 spectra, cast to FP16 in shared memory (up to 64 signals)
cudaError_t launch_xtc32(const XArgs& a, int* d_err, int nsm, cudaStream_t st);
// FP8 form: e4m3 copy of the F16 spectra scaled by 448/absmax per (item = sb*nchan + chan, signal),
// then the e4m3 Gram with the inverse scales applied per product
cudaError_t launch_cast_fp8(const void* spec16, const unsigned* amax, int rows, int nsig, int T, int ts, int nitems,
                            uint8_t* spec8, float* inv_scale, cudaStream_t st);
cudaError_t launch_xtc8(const XArgs& a, int* d_err, int nsm, cudaStream_t st);
size_t xtc_smem_bytes();
cudaError_t launch_unpack_debug(int nchan, const FArgs& a, float* out, cudaStream_t st);
// a bounded device wait that runs out (error word code 6), for tests of the failure path
cudaError_t launch_expire_wait(int* err, cudaStream_t st);
// the same for the tensor-core kernels' mbarrier wait (error word code 7)
cudaError_t launch_expire_wait_tc(int* err, cudaStream_t st);

}  // namespace fx
