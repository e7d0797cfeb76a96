// cueva_stage_hllemc.cu -- stage kernels instantiated for the HLLE flux with
// the second-order MC reconstruction (16_hlle_flow_mcl.f95, flux_solver 3).
// Built twice: plain for the FP64 kernels and with CUEVA_STAGE_MIXED for the
// mixed-precision ones.
#include "cueva_launch.h"
#include "cueva_stage.cuh"

namespace cueva {

CUEVA_STAGE_UNIT(hllemc, 3)

}  // namespace cueva
