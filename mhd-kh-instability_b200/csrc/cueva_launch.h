// cueva_launch.h -- host-side launchers of the kernels in cueva_kernels.cu
#pragma once
#include <cuda_runtime.h>
#include <string>
#include "cueva_common.cuh"
#include "../../include/cueva.h"

struct cueva_mlp;

// records msg as the thread's last error and returns code (cueva_last_error)
int32_t cueva_fail(int32_t code, const std::string& msg);

namespace cueva {
struct MLPDevice;
// the network in the layout the kernels read (host copy), and its device
int32_t mlp_device_image(const cueva_mlp* M, MLPDevice* out);
int mlp_device_of(const cueva_mlp* M);
// sets the shared-memory limits of the stage kernels (call once per device
// before the first launch or capture)
cudaError_t prepare_stage(int rec_mp, int solver, int prec);
// per-solver, per-precision halves of prepare_stage / launch_stage
// (cueva_stage_*.cu; _fp64 plain FP64, _mixed the mixed-precision kernels)
#define CUEVA_DECLARE_STAGE_UNIT(NAME, P)                                                                   \
  cudaError_t prepare_stage_##NAME##_##P(int rec_mp);                                                       \
  cudaError_t launch_stage_##NAME##_##P(int rec_mp, const StageShape& sh, cudaStream_t st, const InstDesc* d, \
                                        int n, const StageArgs& sa, cudaEvent_t* ev);
#define CUEVA_DECLARE_STAGE_SOLVER(NAME) CUEVA_DECLARE_STAGE_UNIT(NAME, fp64) CUEVA_DECLARE_STAGE_UNIT(NAME, mixed)
CUEVA_DECLARE_STAGE_SOLVER(lax)
CUEVA_DECLARE_STAGE_SOLVER(mcl)
CUEVA_DECLARE_STAGE_SOLVER(hllemc)
CUEVA_DECLARE_STAGE_SOLVER(hllcmc)
CUEVA_DECLARE_STAGE_SOLVER(hll)
CUEVA_DECLARE_STAGE_SOLVER(hlle)
CUEVA_DECLARE_STAGE_SOLVER(hllc)
// one RK stage: y faces, then x faces + update; with ev non-null, ev[0..2]
// are recorded before, between and after the launches
cudaError_t launch_stage(int rec_mp, int solver, int prec, const StageShape& sh, cudaStream_t st, const InstDesc* d,
                         int n, const StageArgs& sa, cudaEvent_t* ev = nullptr);
// whether the fused stage kernel k_stage exists for this reconstruction and
// flux routine (tile height FACE_ROWS)
bool stage_fused_available(int rec_mp, int solver);
// grid rows per fused-stage tile for a grid: a multiple of rows, so that the
// launch has enough tiles to balance over `slots` resident CTAs
int stage_seg_rows(int imax, int jmax, int rows, int slots);
cudaError_t launch_begin_step(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur, int qout,
                              double abt11);
cudaError_t launch_startconvar(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur);
cudaError_t launch_electricvarint(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur, int q,
                                  double abtll);
cudaError_t launch_con2prim(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur);
// varfin / electricfield: U += dt * finsum for the conserved slots in mask (bit Q_*)
cudaError_t launch_add_finsum(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur, uint32_t mask);
// 17_fluxandsource.f95 on the stored interface fluxes I.fx / I.fy (FP64): rhs_out of stage sa.l
cudaError_t launch_fluxandsource(long long npts, cudaStream_t st, const InstDesc* d, int n, const StageArgs& sa);
// primitive reconstruction of prim[cur] into prim[1 - cur] + startconvar and
// stage 1 of the reconstructed state (primitive_rec = 1)
cudaError_t launch_recons_begin(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur, int qout,
                                double abt11);
// learned con2prim on the tcgen05 tensor cores after the last stage
// (cueva_c2p.cu): tiles of 128 points per instance, and the launch over
// ntiles tiles of all instances; network seeds of n SoA states
int c2p_tiles(int imax, int jmax);
cudaError_t launch_c2p_step(cudaStream_t st, const InstDesc* d, int ninst, int ntiles, const MLPDevice* mlp, int cur,
                            int qout, double abt11);
cudaError_t launch_predict_tc(long long n, const MLPDevice* mlp, const double* cons, double* pseed,
                              uint32_t* err_status, cudaStream_t st, bool self_test = false);
// run diagnostics of the prims in I.prim[cur] with the given D and tau slabs
// (cueva_diag.cu): diag_blocks() rows of diag_partials() doubles of scratch
int diag_blocks(int imax, int jmax);
int diag_partials();
cudaError_t launch_diag(const InstDesc& I, int cur, const double* D, const double* tau, double b0, double* part,
                        long long h, double t, cueva_diag_record* rec, cudaStream_t st);
}  // namespace cueva
