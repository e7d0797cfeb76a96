// cueva_stage_hll.cu -- stage kernels instantiated for the HLL + MPX (16_hll_flow_mpx.f95)
// solver (one translation unit per solver keeps the builds parallel).
// Built twice: plain for the FP64 kernels and with CUEVA_STAGE_MIXED for the
// mixed-precision ones.
#include "cueva_launch.h"
#include "cueva_stage.cuh"

namespace cueva {

CUEVA_STAGE_UNIT(hll, 5)

}  // namespace cueva
