// fx_fstage_f256.cu -- F-stage kernels for FFT length 256 (see fx_fstage.cuh).
#include <algorithm>

#include "fx_fstage.cuh"

namespace fx {

cudaError_t launch_fstage_256(int mode, const FArgs& a, cudaStream_t st) { return launch_fstage_F<256>(mode, a, st); }

cudaError_t launch_fstage_batch_256(int mode, int npol, int tb, const FArgs* d_jobs, const int4* d_tasks, int ntask,
                                  cudaStream_t st)
{
    return launch_fstage_batch_F<256>(mode, npol, tb, d_jobs, d_tasks, ntask, st);
}

size_t fstage_smem_256(int mode, int tb, int npol) { return fstage_smem<256>(mode, tb, npol); }

}  // namespace fx
