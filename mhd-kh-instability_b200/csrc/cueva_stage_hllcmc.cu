// cueva_stage_hllcmc.cu -- stage kernels instantiated for the HLLC flux with
// the second-order MC reconstruction (16_hllc_flow_mcl.f95, flux_solver 4).
// Built twice: plain for the FP64 kernels and with CUEVA_STAGE_MIXED for the
// mixed-precision ones.
#include "cueva_launch.h"
#include "cueva_stage.cuh"

namespace cueva {

CUEVA_STAGE_UNIT(hllcmc, 4)

}  // namespace cueva
