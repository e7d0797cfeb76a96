// cueva_stage_mcl.cu -- stage kernels instantiated for the HLL flux with the
// second-order MC reconstruction (16_hll_flow_mcl.f95, flux_solver 2).
#include "cueva_launch.h"
#include "cueva_stage.cuh"

namespace cueva {

cudaError_t launch_stage_mcl(int rec_mp, int prec, const StageShape& sh, cudaStream_t st, const InstDesc* d, int n,
                             const StageArgs& sa, cudaEvent_t* ev) {
  return launch_stage_solver<2>(rec_mp, prec, sh, st, d, n, sa, ev);
}

cudaError_t prepare_stage_mcl(int rec_mp, int prec) { return prepare_stage_solver<2>(rec_mp, prec); }

}  // namespace cueva
