// fx_fstage_f4096.cu -- F-stage kernels for FFT length 4096 (see fx_fstage.cuh).
#include <algorithm>

#include "fx_fstage.cuh"

namespace fx {

cudaError_t launch_fstage_4096(int mode, const FArgs& a, cudaStream_t st) { return launch_fstage_F<4096>(mode, a, st); }

cudaError_t launch_fstage_batch_4096(int mode, int npol, int tb, const FArgs* d_jobs, const int4* d_tasks, int ntask,
                                  cudaStream_t st)
{
    return launch_fstage_batch_F<4096>(mode, npol, tb, d_jobs, d_tasks, ntask, st);
}

size_t fstage_smem_4096(int mode, int tb, int npol) { return fstage_smem<4096>(mode, tb, npol); }

}  // namespace fx
