// cueva_stage_lax.cu -- stage kernels instantiated for the Lax-Friedrichs
// flux with MC slopes (15_lax_flow.f95, flux_solver 1).
#include "cueva_launch.h"
#include "cueva_stage.cuh"

namespace cueva {

cudaError_t launch_stage_lax(int rec_mp, int prec, const StageShape& sh, cudaStream_t st, const InstDesc* d, int n,
                             const StageArgs& sa, cudaEvent_t* ev) {
  return launch_stage_solver<1>(rec_mp, prec, sh, st, d, n, sa, ev);
}

cudaError_t prepare_stage_lax(int rec_mp, int prec) { return prepare_stage_solver<1>(rec_mp, prec); }

}  // namespace cueva
