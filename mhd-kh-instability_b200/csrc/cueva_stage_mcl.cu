// cueva_stage_mcl.cu -- stage kernels instantiated for the HLL flux with the
// second-order MC reconstruction (16_hll_flow_mcl.f95, flux_solver 2).
// Built twice: plain for the FP64 kernels and with CUEVA_STAGE_MIXED for the
// mixed-precision ones.
#include "cueva_launch.h"
#include "cueva_stage.cuh"

namespace cueva {

CUEVA_STAGE_UNIT(mcl, 2)

}  // namespace cueva
