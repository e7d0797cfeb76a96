// cueva_launch.h -- host-side launchers of the kernels in cueva_kernels.cu
#pragma once
#include <cuda_runtime.h>
#include "cueva_common.cuh"

namespace cueva {
cudaError_t launch_sweep(int rec_mp, int solver, int prec, int nblocks, cudaStream_t st, const InstDesc* d, int n,
                         const StageArgs& sa);
cudaError_t launch_begin_step(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur, int qout,
                              double abt11);
cudaError_t launch_startconvar(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur);
cudaError_t launch_electricvarint(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur, int q,
                                  double abtll);
cudaError_t launch_con2prim(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur);
}  // namespace cueva
