// fx_fstage_f8192.cu -- F-stage kernels for FFT length 8192 (see fx_fstage.cuh).
#include <algorithm>

#include "fx_fstage.cuh"

namespace fx {

cudaError_t launch_fstage_8192(int mode, const FArgs& a, cudaStream_t st) { return launch_fstage_F<8192>(mode, a, st); }

cudaError_t launch_fstage_batch_8192(int mode, int npol, int tb, const FArgs* d_jobs, const int4* d_tasks, int ntask,
                                  cudaStream_t st)
{
    return launch_fstage_batch_F<8192>(mode, npol, tb, d_jobs, d_tasks, ntask, st);
}

size_t fstage_smem_8192(int mode, int tb, int npol) { return fstage_smem<8192>(mode, tb, npol); }

}  // namespace fx
