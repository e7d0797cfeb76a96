// cueva_kernels.cu -- pointwise kernels of the CUEVA hot path (begin of
// step, routine mirrors) and the dispatch of the stage launches to the
// per-solver translation units (cueva_stage_{hll,hllc,hlle}.cu; the stage
// kernels themselves are described in cueva_stage.cuh).
#include "cueva_launch.h"
#include "cueva_stage.cuh"

namespace cueva {

// ------------------------------------------------------------ prologue
// startconvar + stage-1 state for the prims in prim[cur]
__global__ void k_begin_step(const InstDesc* __restrict__ insts, int ninst, int cur, int qout, double abt11) {
  const InstDesc& I = insts[blockIdx.y];
  const int nx = I.imax + 1, ny = I.jmax + 1;
  const long long fs = I.fstride;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nx * ny;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = int(t % nx), j = int(t / nx);
    const long long pc = (long long)j * I.pitch + i;
    double pv[NPRIM];
#pragma unroll
    for (int c = 0; c < NPRIM; ++c) pv[c] = I.prim[cur][c * fs + pc];
    begin_step_point(I, abt11, I.aux[cur], I.stage[qout], pc, pv);
  }
  (void)ninst;
}

// primitive reconstruction (05_reconstruct.f95:525-746, primitive_rec = 1):
// per field, the monotonized-central slope along the grid diagonal
// (limit = 2, funciones.f95:104-147), L = u + x and R = u - x with
// x = slope / 2 (both faces of a point take the same slope arguments), and
// the new value (R + L) / 2; ghost points by the boundary maps.  Reads
// prim[cur], writes the reconstructed primitives to prim[1 - cur] and
// prepares the step from them (startconvar, stage 1).
__device__ __forceinline__ double limiter_mc(double ga, double gb) {
  return 0.5 * (fsgn1(ga) + fsgn1(gb)) *
         fmin2(fmin2(2.0 * fabs(ga), 2.0 * fabs(gb)), 0.5 * fabs(ga + gb));
}

__global__ void k_recons_begin(const InstDesc* __restrict__ insts, int cur, int qout, double abt11) {
  const InstDesc& I = insts[blockIdx.y];
  if (!I.primitive_rec) return;
  const int nx = I.imax + 1, ny = I.jmax + 1;
  const long long fs = I.fstride;
  const double* u = I.prim[cur];
  double* un = I.prim[1 - cur];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nx * ny;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = int(t % nx), j = int(t / nx);
    const long long pc = (long long)j * I.pitch + i;
    const long long pm = (long long)map_idx(j - 1, I.jmax, I.bc_y) * I.pitch + map_idx(i - 1, I.imax, I.bc_x);
    const long long pp = (long long)map_idx(j + 1, I.jmax, I.bc_y) * I.pitch + map_idx(i + 1, I.imax, I.bc_x);
    double pv[NPRIM];
#pragma unroll
    for (int c = 0; c < NPRIM; ++c) {
      const double m1 = u[c * fs + pm], m = u[c * fs + pc], p1 = u[c * fs + pp];
      const double x = 0.5 * limiter_mc(p1 - m, m - m1);
      pv[c] = 0.5 * ((m - x) + (m + x));
      un[c * fs + pc] = pv[c];
    }
    begin_step_point(I, abt11, I.aux[1 - cur], I.stage[qout], pc, pv);
  }
}

// ------------------------------------------------- routine mirrors (pointwise)
// startconvar only (06_conserved_var.f95:79-140)
__global__ void k_startconvar(const InstDesc* __restrict__ insts, int cur) {
  const InstDesc& I = insts[blockIdx.y];
  const int nx = I.imax + 1, ny = I.jmax + 1;
  const long long fs = I.fstride;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nx * ny;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = int(t % nx), j = int(t / nx);
    const long long pc = (long long)j * I.pitch + i;
    const double* p = I.prim[cur];
    const Cons c = startconvar(p[P_RHO * fs + pc], p[P_P * fs + pc], p[P_VX * fs + pc], p[P_VY * fs + pc],
                               p[P_VZ * fs + pc], p[P_EX * fs + pc], p[P_EY * fs + pc], p[P_EZ * fs + pc],
                               p[P_BX * fs + pc], p[P_BY * fs + pc], p[P_BZ * fs + pc], I.gamma);
    double* a = I.aux[cur];
    a[A_D * fs + pc] = c.D; a[A_TAU * fs + pc] = c.tau; a[A_SX * fs + pc] = c.Sx;
    a[A_SY * fs + pc] = c.Sy; a[A_SZ * fs + pc] = c.Sz; a[A_W * fs + pc] = c.W;
  }
}

// electricvarint for stage l (11_elecvarint.f95:279-328) followed by the
// current of flowinit (14_flowinit.f95:280-302): reads E* from the E slots
// of stage[q], overwrites them with E_l and fills J
__global__ void k_electricvarint(const InstDesc* __restrict__ insts, int cur, int q, double abtll) {
  const InstDesc& I = insts[blockIdx.y];
  const int nx = I.imax + 1, ny = I.jmax + 1;
  const long long fs = I.fstride;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nx * ny;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = int(t % nx), j = int(t / nx);
    const long long pc = (long long)j * I.pitch + i;
    const double* p = I.prim[cur];
    double* Q = I.stage[q];
    const double W = I.aux[cur][A_W * fs + pc];
    const double vx = p[P_VX * fs + pc], vy = p[P_VY * fs + pc], vz = p[P_VZ * fs + pc];
    const double Bx = Q[Q_BX * fs + pc], By = Q[Q_BY * fs + pc], Bz = Q[Q_BZ * fs + pc];
    double Ex, Ey, Ez;
    implicit_e(abtll, I.sigma, I.dt, W, vx, vy, vz, Bx, By, Bz, Q[Q_EX * fs + pc], Q[Q_EY * fs + pc],
               Q[Q_EZ * fs + pc], Ex, Ey, Ez);
    double Jx, Jy, Jz;
    current(I.sigma, W, vx, vy, vz, Ex, Ey, Ez, Bx, By, Bz, Q[Q_Q * fs + pc], Jx, Jy, Jz);
    Q[Q_EX * fs + pc] = Ex; Q[Q_EY * fs + pc] = Ey; Q[Q_EZ * fs + pc] = Ez;
    Q[Q_JX * fs + pc] = Jx; Q[Q_JY * fs + pc] = Jy; Q[Q_JZ * fs + pc] = Jz;
  }
}

// 17_fluxandsource.f95:433-699 on stored interface fluxes (the routine
// mirror cueva_fluxandsource): Fx(i+1/2, j) in I.fx and Fy(i, j+1/2) in I.fy,
// both FP64; the x differences are formed as in k_xupd, the rest is the same
// update_point, so the result equals the fused stage's right-hand side
__global__ void k_fluxandsource(const InstDesc* __restrict__ insts, StageArgs sa) {
  const InstDesc& I = insts[blockIdx.y];
  const int nx = I.imax + 1, ny = I.jmax + 1;
  const long long fs = I.fstride;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nx * ny;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = int(t % nx), j = int(t / nx);
    const long long pc = (long long)j * I.pitch + i, fo = (long long)j * I.fpitch + i + 1;
    double qx[NROLE];
#pragma unroll
    for (int c = 0; c < NROLE; ++c) {
      const double d = I.fx[c * I.ffs + fo] - I.fx[c * I.ffs + fo - 1];
      qx[c] = I.inv_delx_pow2 != 0.0 ? d * I.inv_delx_pow2 : d / I.delx;
    }
    const double* Q = I.stage[sa.qin];
    const double* pv = I.prim[sa.cur];
    const Centre cv{Q[Q_Q * fs + pc], Q[Q_PSI * fs + pc], Q[Q_PHI * fs + pc], Q[Q_EX * fs + pc],
                    Q[Q_EY * fs + pc], Q[Q_EZ * fs + pc], Q[Q_BX * fs + pc], Q[Q_BY * fs + pc],
                    Q[Q_BZ * fs + pc], pv[P_VX * fs + pc], pv[P_VY * fs + pc], pv[P_VZ * fs + pc]};
    const long long fyo = (long long)(j + 1) * I.fpitch + i;
    auto fyd = [&](int r) { return I.fy[r * I.ffs + fyo] - I.fy[r * I.ffs + fyo - I.fpitch]; };
    const uint32_t st = update_point<EP_RHS, double, 0>(I, sa, i, j, qx, fyd, cv);
    if (st) atomicOr(I.status, st);
  }
}

// varfin / electricfield (19_varfin.f95:16-54, 20_electricfield.f95:153-167):
// U += dt * finsum for the conserved slots of mask (bit Q_*), U being the
// carried primitive (psi, phi, E, B, q) or the time-n conserved (D, tau, S)
__global__ void k_add_finsum(const InstDesc* __restrict__ insts, int cur, uint32_t mask) {
  const InstDesc& I = insts[blockIdx.y];
  const int nx = I.imax + 1, ny = I.jmax + 1;
  const long long fs = I.fstride;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nx * ny;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = int(t % nx), j = int(t / nx);
    const long long pc = (long long)j * I.pitch + i;
#pragma unroll
    for (int c = 0; c < NCONS; ++c) {
      if (!(mask >> c & 1u)) continue;
      double* u = (c < Q_D) ? I.prim[cur] + (long long)(c == Q_PSI ? P_PSI : c == Q_PHI ? P_PHI
                                                          : c <= Q_EZ ? P_EX + (c - Q_EX)
                                                          : c <= Q_BZ ? P_BX + (c - Q_BX) : P_Q) * fs
                            : I.aux[cur] + (long long)(A_D + (c - Q_D)) * fs;
      u[pc] = u[pc] + I.dt * I.finsum[c * fs + pc];
    }
  }
}

// con2prim with l_swap = 1: the evolved D, tau, S in aux[cur] and E, B in
// prim[cur]; seeds v, rho, p are the prims in prim[cur]; result overwrites prim[cur]
__global__ void k_con2prim(const InstDesc* __restrict__ insts, int cur) {
  const InstDesc& I = insts[blockIdx.y];
  const int nx = I.imax + 1, ny = I.jmax + 1;
  const long long fs = I.fstride;
  uint32_t st = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nx * ny;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = int(t % nx), j = int(t / nx);
    const long long pc = (long long)j * I.pitch + i;
    double* p = I.prim[cur];
    const double* a = I.aux[cur];
    C2PIn in{a[A_D * fs + pc], a[A_TAU * fs + pc], a[A_SX * fs + pc], a[A_SY * fs + pc], a[A_SZ * fs + pc],
             p[P_EX * fs + pc], p[P_EY * fs + pc], p[P_EZ * fs + pc], p[P_BX * fs + pc], p[P_BY * fs + pc],
             p[P_BZ * fs + pc], p[P_VX * fs + pc], p[P_VY * fs + pc], p[P_VZ * fs + pc], p[P_RHO * fs + pc],
             p[P_P * fs + pc]};
    C2POut o;
    st |= c2p_dispatch(I, in, o);
    p[P_VX * fs + pc] = o.vx; p[P_VY * fs + pc] = o.vy; p[P_VZ * fs + pc] = o.vz;
    p[P_RHO * fs + pc] = o.rho; p[P_P * fs + pc] = o.p;
  }
  if (st) atomicOr(I.status, st);
}

// ------------------------------------------------------------- dispatch
bool stage_fused_available(int rec_mp, int solver) {
  const int rm = solver <= 4 ? 3 : rec_mp;   // the flux routines 1-4 use the MC slopes
  switch (rm) {
    case 0: return kFused<0>;
    case 1: return kFused<1>;
    case 2: return kFused<2>;
    case 3: return kFused<3>;
    default: return false;
  }
}

int stage_seg_rows(int imax, int jmax, int rows, int slots) {
  // A tile of nb bands updates nb * rows - 1 grid rows (its first band also
  // computes the faces below the segment) and costs about nb band times; the
  // launch takes about ceil(tiles / slots) tile times.  Pick the band count
  // with the smallest product (the larger one on ties: fewer repeated faces).
  const int strips = (imax + 1 + 30) / 31;
  int best = 1;
  long long best_cost = -1;
  for (int nb = 1; nb <= 32; ++nb) {
    const int seg = nb * rows - 1;
    const long long tiles = (long long)strips * ((jmax + 1 + seg - 1) / seg);
    const long long cost = (tiles + slots - 1) / slots * nb;
    if (best_cost < 0 || cost <= best_cost) { best_cost = cost; best = nb; }
  }
  return best * rows - 1;
}

cudaError_t prepare_stage(int rec_mp, int solver, int prec) {
#define CUEVA_PREPARE_CASE(K, NAME) \
  case K: return prec ? prepare_stage_##NAME##_mixed(rec_mp) : prepare_stage_##NAME##_fp64(rec_mp);
  switch (solver) {
    CUEVA_PREPARE_CASE(1, lax)
    CUEVA_PREPARE_CASE(2, mcl)
    CUEVA_PREPARE_CASE(3, hllemc)
    CUEVA_PREPARE_CASE(4, hllcmc)
    CUEVA_PREPARE_CASE(5, hll)
    CUEVA_PREPARE_CASE(6, hlle)
    CUEVA_PREPARE_CASE(7, hllc)
    default: return cudaErrorInvalidValue;
  }
#undef CUEVA_PREPARE_CASE
}

cudaError_t launch_stage(int rec_mp, int solver, int prec, const StageShape& sh, cudaStream_t st, const InstDesc* d,
                         int n, const StageArgs& sa, cudaEvent_t* ev) {
#define CUEVA_LAUNCH_CASE(K, NAME)                                                 \
  case K:                                                                        \
    return prec ? launch_stage_##NAME##_mixed(rec_mp, sh, st, d, n, sa, ev)      \
                : launch_stage_##NAME##_fp64(rec_mp, sh, st, d, n, sa, ev);
  switch (solver) {
    CUEVA_LAUNCH_CASE(1, lax)
    CUEVA_LAUNCH_CASE(2, mcl)
    CUEVA_LAUNCH_CASE(3, hllemc)
    CUEVA_LAUNCH_CASE(4, hllcmc)
    CUEVA_LAUNCH_CASE(5, hll)
    CUEVA_LAUNCH_CASE(6, hlle)
    CUEVA_LAUNCH_CASE(7, hllc)
    default: return cudaErrorInvalidValue;
  }
#undef CUEVA_LAUNCH_CASE
}

static dim3 point_grid(long long npts, int ninst) {
  long long b = (npts + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return dim3((unsigned)b, (unsigned)ninst);
}

cudaError_t launch_begin_step(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur, int qout,
                              double abt11) {
  k_begin_step<<<point_grid(npts, n), 256, 0, st>>>(d, n, cur, qout, abt11);
  return cudaGetLastError();
}
cudaError_t launch_startconvar(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur) {
  k_startconvar<<<point_grid(npts, n), 256, 0, st>>>(d, cur);
  return cudaGetLastError();
}
cudaError_t launch_electricvarint(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur, int q,
                                  double abtll) {
  k_electricvarint<<<point_grid(npts, n), 256, 0, st>>>(d, cur, q, abtll);
  return cudaGetLastError();
}
cudaError_t launch_recons_begin(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur, int qout,
                                double abt11) {
  k_recons_begin<<<point_grid(npts, n), 256, 0, st>>>(d, cur, qout, abt11);
  return cudaGetLastError();
}
cudaError_t launch_fluxandsource(long long npts, cudaStream_t st, const InstDesc* d, int n, const StageArgs& sa) {
  k_fluxandsource<<<point_grid(npts, n), 256, 0, st>>>(d, sa);
  return cudaGetLastError();
}
cudaError_t launch_add_finsum(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur, uint32_t mask) {
  k_add_finsum<<<point_grid(npts, n), 256, 0, st>>>(d, cur, mask);
  return cudaGetLastError();
}
cudaError_t launch_con2prim(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur) {
  k_con2prim<<<point_grid(npts, n), 256, 0, st>>>(d, cur);
  return cudaGetLastError();
}

}  // namespace cueva

