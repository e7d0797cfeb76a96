// cueva_stage_hllc.cu -- stage kernels instantiated for the HLLC + MPX (16_hllc_flow_mpx.f95)
// solver (one translation unit per solver keeps the builds parallel).
#include "cueva_launch.h"
#include "cueva_stage.cuh"

namespace cueva {

cudaError_t launch_stage_hllc(int rec_mp, int prec, const StageShape& sh, cudaStream_t st, const InstDesc* d, int n,
                              const StageArgs& sa, cudaEvent_t* ev) {
  return launch_stage_solver<7>(rec_mp, prec, sh, st, d, n, sa, ev);
}

cudaError_t prepare_stage_hllc(int rec_mp, int prec) { return prepare_stage_solver<7>(rec_mp, prec); }

}  // namespace cueva
