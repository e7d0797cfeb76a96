// cueva_stage_hllc.cu -- stage kernels instantiated for the HLLC + MPX (16_hllc_flow_mpx.f95)
// solver (one translation unit per solver keeps the builds parallel).
// Built twice: plain for the FP64 kernels and with CUEVA_STAGE_MIXED for the
// mixed-precision ones.
#include "cueva_launch.h"
#include "cueva_stage.cuh"

namespace cueva {

CUEVA_STAGE_UNIT(hllc, 7)

}  // namespace cueva
