// cueva_stage_lax.cu -- stage kernels instantiated for the Lax-Friedrichs
// flux with MC slopes (15_lax_flow.f95, flux_solver 1).
// Built twice: plain for the FP64 kernels and with CUEVA_STAGE_MIXED for the
// mixed-precision ones.
#include "cueva_launch.h"
#include "cueva_stage.cuh"

namespace cueva {

CUEVA_STAGE_UNIT(lax, 1)

}  // namespace cueva
