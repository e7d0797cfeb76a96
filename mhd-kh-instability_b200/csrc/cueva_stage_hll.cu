// cueva_stage_hll.cu -- stage kernels instantiated for the HLL + MPX (16_hll_flow_mpx.f95)
// solver (one translation unit per solver keeps the builds parallel).
#include "cueva_launch.h"
#include "cueva_stage.cuh"

namespace cueva {

cudaError_t launch_stage_hll(int rec_mp, int prec, const StageShape& sh, cudaStream_t st, const InstDesc* d, int n,
                              const StageArgs& sa, cudaEvent_t* ev) {
  return launch_stage_solver<5>(rec_mp, prec, sh, st, d, n, sa, ev);
}

cudaError_t prepare_stage_hll(int rec_mp, int prec) { return prepare_stage_solver<5>(rec_mp, prec); }

}  // namespace cueva
