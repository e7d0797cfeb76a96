// cueva_stage_hllemc.cu -- stage kernels instantiated for the HLLE flux with
// the second-order MC reconstruction (16_hlle_flow_mcl.f95, flux_solver 3).
#include "cueva_launch.h"
#include "cueva_stage.cuh"

namespace cueva {

cudaError_t launch_stage_hllemc(int rec_mp, int prec, const StageShape& sh, cudaStream_t st, const InstDesc* d,
                                int n, const StageArgs& sa, cudaEvent_t* ev) {
  return launch_stage_solver<3>(rec_mp, prec, sh, st, d, n, sa, ev);
}

cudaError_t prepare_stage_hllemc(int rec_mp, int prec) { return prepare_stage_solver<3>(rec_mp, prec); }

}  // namespace cueva
