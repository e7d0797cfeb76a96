// cueva_stage_hllcmc.cu -- stage kernels instantiated for the HLLC flux with
// the second-order MC reconstruction (16_hllc_flow_mcl.f95, flux_solver 4).
#include "cueva_launch.h"
#include "cueva_stage.cuh"

namespace cueva {

cudaError_t launch_stage_hllcmc(int rec_mp, int prec, const StageShape& sh, cudaStream_t st, const InstDesc* d,
                                int n, const StageArgs& sa, cudaEvent_t* ev) {
  return launch_stage_solver<4>(rec_mp, prec, sh, st, d, n, sa, ev);
}

cudaError_t prepare_stage_hllcmc(int rec_mp, int prec) { return prepare_stage_solver<4>(rec_mp, prec); }

}  // namespace cueva
