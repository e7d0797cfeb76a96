// cueva_kernels.cu -- sm_100a kernels of the CUEVA per-step hot path.
//
// One RK stage = one launch of k_sweep.  A warp owns a strip of 32 grid
// points (31 output cells + one halo column on the left) and marches up a
// block of SWEEP_ROWS rows.  At every point (i, j) the thread does exactly
// the work of one iteration of the reference's Riemann loop
// (16_hll_flow_mpx.f95:1358-1965 / 16_hllc_flow_mpx.f95:2401-4618): it
// reconstructs the x interface i+1/2 and the y interface j+1/2 with MP5/7/9
// (its own registers, loads through L1), applies the superluminal fall-back
// that couples the two directions, and solves both Riemann problems.  The
// x-flux of the neighbour interface i-1/2 arrives by warp shuffle, the
// y-flux of j-1/2 is the thread's own result from the previous row, so the
// flux divergence (17_fluxandsource.f95:441-635) needs no shared memory and
// no flux array ever touches HBM.  The epilogue is pointwise and fused:
// sumfin, the next stage's sumint/varint/electricvarint/flowinit, or - after
// the last stage - varfin/electricfield, con2prim and the next step's
// startconvar.
#include <cuda_runtime.h>
#include <math_constants.h>

#include "cueva_common.cuh"
#include "cueva_mp.cuh"
#include "cueva_riemann.cuh"
#include "cueva_point.cuh"
#include "cueva_mlp.cuh"

namespace cueva {

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ const InstDesc& find_inst(const InstDesc* __restrict__ insts, int ninst, int b) {
  int k = 0;
  for (int t = 1; t < ninst; ++t)
    if (insts[t].block_begin <= b) k = t;
  return insts[k];
}

template <typename T>
__device__ __forceinline__ T ldT(const double* p) { return T(__ldg(p)); }

// begin-of-step work for one interior point: startconvar of the new prims,
// stage-1 state Q_1 = U + dt*0 (cleanvarint zeroed intsum), its implicit E
// and current J (06_conserved_var.f95, 10_varint.f95, 11_elecvarint.f95,
// 14_flowinit.f95 for l = 1)
__device__ __forceinline__ void begin_step_point(const InstDesc& I, double abt11, double* auxo, double* Qo,
                                                 long long pc, const double* pv) {
  const long long fs = I.fstride;
  const Cons c = startconvar(pv[P_RHO], pv[P_P], pv[P_VX], pv[P_VY], pv[P_VZ], pv[P_EX], pv[P_EY], pv[P_EZ],
                             pv[P_BX], pv[P_BY], pv[P_BZ], I.gamma);
  auxo[A_D * fs + pc] = c.D;
  auxo[A_TAU * fs + pc] = c.tau;
  auxo[A_SX * fs + pc] = c.Sx;
  auxo[A_SY * fs + pc] = c.Sy;
  auxo[A_SZ * fs + pc] = c.Sz;
  auxo[A_W * fs + pc] = c.W;
  const double z = I.dt * 0.0;
  const double Bx = pv[P_BX] + z, By = pv[P_BY] + z, Bz = pv[P_BZ] + z, q = pv[P_Q] + z;
  double Ex, Ey, Ez;
  implicit_e(abt11, I.sigma, I.dt, c.W, pv[P_VX], pv[P_VY], pv[P_VZ], Bx, By, Bz, pv[P_EX] + z, pv[P_EY] + z,
             pv[P_EZ] + z, Ex, Ey, Ez);
  double Jx, Jy, Jz;
  current(I.sigma, c.W, pv[P_VX], pv[P_VY], pv[P_VZ], Ex, Ey, Ez, Bx, By, Bz, q, Jx, Jy, Jz);
  Qo[Q_PSI * fs + pc] = pv[P_PSI] + z;
  Qo[Q_PHI * fs + pc] = pv[P_PHI] + z;
  Qo[Q_EX * fs + pc] = Ex;
  Qo[Q_EY * fs + pc] = Ey;
  Qo[Q_EZ * fs + pc] = Ez;
  Qo[Q_BX * fs + pc] = Bx;
  Qo[Q_BY * fs + pc] = By;
  Qo[Q_BZ * fs + pc] = Bz;
  Qo[Q_Q * fs + pc] = q;
  Qo[Q_D * fs + pc] = c.D + z;
  Qo[Q_TAU * fs + pc] = c.tau + z;
  Qo[Q_SX * fs + pc] = c.Sx + z;
  Qo[Q_SY * fs + pc] = c.Sy + z;
  Qo[Q_SZ * fs + pc] = c.Sz + z;
  Qo[Q_JX * fs + pc] = Jx;
  Qo[Q_JY * fs + pc] = Jy;
  Qo[Q_JZ * fs + pc] = Jz;
}

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

// con2prim with l_swap = 1: the evolved D, tau, S in aux[cur] and E, B in
// prim[cur]; seeds v, rho, p are the prims in prim[cur]; result overwrites prim[cur]
__device__ __forceinline__ uint32_t c2p_dispatch(const InstDesc& I, const C2PIn& in, C2POut& o) {
  if (I.c2p == 1) return c2p_cardano(in, I.gamma, I.eps1_c2p, o, I.counters);
  if (I.c2p == 0) return c2p_nr(in, I.gamma, o);
  return c2p_learned(in, I.gamma, I.eps1_c2p, I.mlp, o, I.counters);
}

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

// -------------------------------------------------------------- the sweep
template <int RM, int SOLVER, typename T>
struct Sweep {
  static constexpr int R = MPR<RM>::R;
  static constexpr int NS = 2 * R + 2;
};

template <int RM, int SOLVER, typename T>
__global__ void __launch_bounds__(SWEEP_WARPS * 32)
k_sweep(const InstDesc* __restrict__ insts, int ninst, StageArgs sa) {
  constexpr int R = MPR<RM>::R;
  constexpr int NS = 2 * R + 2;
  const InstDesc& I = find_inst(insts, ninst, blockIdx.x);
  const int lb = blockIdx.x - I.block_begin;
  const int bx_per = (I.strips_x + SWEEP_WARPS - 1) / SWEEP_WARPS;
  const int bx = lb % bx_per, by = lb / bx_per;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sx = bx * SWEEP_WARPS + warp;
  if (sx >= I.strips_x) return;   // warp-uniform

  const int imax = I.imax, jmax = I.jmax, pitch = I.pitch, bcx = I.bc_x, bcy = I.bc_y;
  const long long fs = I.fstride;
  const T gamma = T(I.gamma);
  const int i = sx * STRIP - 1 + lane;            // this thread's point column
  const bool col_ok = (i <= imax);
  const bool out_col = col_ok && lane >= 1;
  const int j0 = by * SWEEP_ROWS;
  const int j1 = min(j0 + SWEEP_ROWS - 1, jmax);
  const double* __restrict__ prim = I.prim[sa.cur];
  const double* __restrict__ aux = I.aux[sa.cur];
  const double* __restrict__ Q = I.stage[sa.qin];

  const int ic = min(i, imax);
  int colx[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) colx[k] = map_idx(ic - R + k, imax, bcx);
  const int ci = map_idx(ic, imax, bcx), cim1 = map_idx(ic - 1, imax, bcx);

  T prevFy[NROLE];
#pragma unroll
  for (int c = 0; c < NROLE; ++c) prevFy[c] = T(0);

  for (int jj = j0 - 1; jj <= j1; ++jj) {
    const bool halo = (jj == j0 - 1);
    T Fx[NROLE], Fy[NROLE];
#pragma unroll
    for (int c = 0; c < NROLE; ++c) { Fx[c] = T(0); Fy[c] = T(0); }
    uint32_t st = 0;
    if (col_ok) {
      const int rj = map_idx(jj, jmax, bcy);
      const int rjm1 = map_idx(jj - 1, jmax, bcy);
      const long long rowx = (long long)rj * pitch;
      long long rowy[NS];
#pragma unroll
      for (int k = 0; k < NS; ++k) rowy[k] = (long long)map_idx(jj - R + k, jmax, bcy) * pitch;

      auto rx = [&](const double* f, T& L, T& Rv) {
        T u[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) u[k] = ldT<T>(f + rowx + colx[k]);
        mp_pair<RM>(u, L, Rv);
      };
      auto ry = [&](const double* f, T& L, T& Rv) {
        T u[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) u[k] = ldT<T>(f + rowy[k] + ci);
        mp_pair<RM>(u, L, Rv);
      };
      auto rxp = [&](const double* f, T& L, T& Rv) {
        T u[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) u[k] = ldT<T>(f + rowx + colx[k]);
        mp_pair_pos<RM>(u, L, Rv);
      };
      auto ryp = [&](const double* f, T& L, T& Rv) {
        T u[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) u[k] = ldT<T>(f + rowy[k] + ci);
        mp_pair_pos<RM>(u, L, Rv);
      };

      Side<T> xl, xr, yl, yr;
      // primitive slots 21-25 (x) and 58-62 (y) of 16_hll_flow_mpx.f95
      rx(prim + P_VX * fs, xl.vx, xr.vx); rx(prim + P_VY * fs, xl.vy, xr.vy); rx(prim + P_VZ * fs, xl.vz, xr.vz);
      ry(prim + P_VX * fs, yl.vx, yr.vx); ry(prim + P_VY * fs, yl.vy, yr.vy); ry(prim + P_VZ * fs, yl.vz, yr.vz);
      rxp(prim + P_P * fs, xl.p, xr.p); rxp(prim + P_RHO * fs, xl.rho, xr.rho);
      ryp(prim + P_P * fs, yl.p, yr.p); ryp(prim + P_RHO * fs, yl.rho, yr.rho);

      if constexpr (SOLVER == 5 || SOLVER == 7) {
        // superluminal fall-back to cell velocities, 16_hll_flow_mpx.f95:1393-1462
        // (the right states take cells i-1 / j-1, as in the reference)
        const T V2xl = pw2(xl.vx) + pw2(xl.vy) + pw2(xl.vz);
        const T V2xr = pw2(xr.vx) + pw2(xr.vy) + pw2(xr.vz);
        const T V2yl = pw2(yl.vx) + pw2(yl.vy) + pw2(yl.vz);
        const T V2yr = pw2(yr.vx) + pw2(yr.vy) + pw2(yr.vz);
        if (V2xl >= T(1) || V2xr >= T(1) || V2yl >= T(1) || V2yr >= T(1)) {
          const long long c0 = rowx + ci, cmx = rowx + cim1, cmy = (long long)rjm1 * pitch + ci;
          xl.vx = yl.vx = ldT<T>(prim + P_VX * fs + c0);
          xl.vy = yl.vy = ldT<T>(prim + P_VY * fs + c0);
          xl.vz = yl.vz = ldT<T>(prim + P_VZ * fs + c0);
          xr.vx = ldT<T>(prim + P_VX * fs + cmx); xr.vy = ldT<T>(prim + P_VY * fs + cmx);
          xr.vz = ldT<T>(prim + P_VZ * fs + cmx);
          yr.vx = ldT<T>(prim + P_VX * fs + cmy); yr.vy = ldT<T>(prim + P_VY * fs + cmy);
          yr.vz = ldT<T>(prim + P_VZ * fs + cmy);
        }
      }
      if constexpr (SOLVER == 7) {
        // density fix-up chain, 16_hllc_flow_mpx.f95:2663-2690 (time-n rho of the cell)
        if (yl.rho < T(0) || yr.rho < T(0) || xl.rho < T(0) || xr.rho < T(0)) {
          const T r10 = T(__ldg(prim + P_RHO * fs + rowx + ci) * 1.0e-1);
          if (yl.rho < T(0)) yl.rho = r10;
          else if (yr.rho < T(0)) yr.rho = r10;
          else if (xl.rho < T(0)) xl.rho = r10;
          else xr.rho = r10;
        }
      }

      if (!halo) {
        rx(Q + Q_PSI * fs, xl.psi, xr.psi); rx(Q + Q_PHI * fs, xl.phi, xr.phi);
        rx(Q + Q_EX * fs, xl.Ex, xr.Ex); rx(Q + Q_EY * fs, xl.Ey, xr.Ey); rx(Q + Q_EZ * fs, xl.Ez, xr.Ez);
        rx(Q + Q_BX * fs, xl.Bx, xr.Bx); rx(Q + Q_BY * fs, xl.By, xr.By); rx(Q + Q_BZ * fs, xl.Bz, xr.Bz);
        rx(Q + Q_Q * fs, xl.q, xr.q); rx(Q + Q_D * fs, xl.D, xr.D); rx(Q + Q_TAU * fs, xl.tau, xr.tau);
        rx(Q + Q_SX * fs, xl.Sx, xr.Sx); rx(Q + Q_SY * fs, xl.Sy, xr.Sy); rx(Q + Q_SZ * fs, xl.Sz, xr.Sz);
        rx(Q + Q_JX * fs, xl.J, xr.J);
        if constexpr (SOLVER == 5) hll_fluxes<0>(xl, xr, gamma, Fx);
        else hllc_fluxes<0>(xl, xr, gamma, Fx, st);
      }
      ry(Q + Q_PSI * fs, yl.psi, yr.psi); ry(Q + Q_PHI * fs, yl.phi, yr.phi);
      ry(Q + Q_EX * fs, yl.Ex, yr.Ex); ry(Q + Q_EY * fs, yl.Ey, yr.Ey); ry(Q + Q_EZ * fs, yl.Ez, yr.Ez);
      ry(Q + Q_BX * fs, yl.Bx, yr.Bx); ry(Q + Q_BY * fs, yl.By, yr.By); ry(Q + Q_BZ * fs, yl.Bz, yr.Bz);
      ry(Q + Q_Q * fs, yl.q, yr.q); ry(Q + Q_D * fs, yl.D, yr.D); ry(Q + Q_TAU * fs, yl.tau, yr.tau);
      ry(Q + Q_SX * fs, yl.Sx, yr.Sx); ry(Q + Q_SY * fs, yl.Sy, yr.Sy); ry(Q + Q_SZ * fs, yl.Sz, yr.Sz);
      ry(Q + Q_JY * fs, yl.J, yr.J);
      if constexpr (SOLVER == 5) hll_fluxes<1>(yl, yr, gamma, Fy);
      else hllc_fluxes<1>(yl, yr, gamma, Fy, st);
    }
    // x flux of the interface i-1/2 from the left neighbour lane
    T Fw[NROLE];
#pragma unroll
    for (int c = 0; c < NROLE; ++c) Fw[c] = __shfl_up_sync(0xffffffffu, Fx[c], 1);

    if (!halo && out_col) {
      const long long pc = (long long)jj * pitch + i;
      const double dlx = I.delx, dly = I.dely;
      auto dxv = [&](int r) { return double(Fx[r]) - double(Fw[r]); };
      auto dyv = [&](int r) { return double(Fy[r]) - double(prevFy[r]); };
      // centre values of stage l and time n
      const double q = Q[Q_Q * fs + pc], psi = Q[Q_PSI * fs + pc], phi = Q[Q_PHI * fs + pc];
      const double Ex = Q[Q_EX * fs + pc], Ey = Q[Q_EY * fs + pc], Ez = Q[Q_EZ * fs + pc];
      const double Bx = Q[Q_BX * fs + pc], By = Q[Q_BY * fs + pc], Bz = Q[Q_BZ * fs + pc];
      const double vx = prim[P_VX * fs + pc], vy = prim[P_VY * fs + pc], vz = prim[P_VZ * fs + pc];
      const double W = aux[A_W * fs + pc];
      double K[NRHS];
      // 17_fluxandsource.f95:488-598; z differences are (X - X)/Delz = 0
      K[Q_PSI] = -(dxv(R_PSI)) / dlx - (dyv(R_PSI)) / dly + q - I.kappa_psi * psi;
      K[Q_PHI] = -(dxv(R_PHI)) / dlx - (dyv(R_PHI)) / dly - I.kappa_phi * phi;
      K[Q_BX] = -(dyv(R_BT2)) / dly + 0.0 - (dxv(R_BN)) / dlx;
      K[Q_BY] = (dxv(R_BT1)) / dlx - (dyv(R_BN)) / dly;
      K[Q_BZ] = -(dxv(R_BT2)) / dlx + (dyv(R_BT1)) / dly;
      K[Q_EX] = (dyv(R_ET2)) / dly - (dxv(R_EN)) / dlx - q * vx;
      K[Q_EY] = 0.0 - (dxv(R_ET1)) / dlx - (dyv(R_EN)) / dly - q * vy;
      K[Q_EZ] = (dxv(R_ET2)) / dlx - (dyv(R_ET1)) / dly - q * vz;
      K[Q_Q] = -(dxv(R_Q)) / dlx - (dyv(R_Q)) / dly;
      K[Q_D] = -(dxv(R_D)) / dlx - (dyv(R_D)) / dly;
      K[Q_TAU] = -(dxv(R_TAU)) / dlx - (dyv(R_TAU)) / dly;
      K[Q_SX] = -(dxv(R_SN)) / dlx - (dyv(R_ST2)) / dly;
      K[Q_SY] = -(dxv(R_ST1)) / dlx - (dyv(R_SN)) / dly;
      K[Q_SZ] = -(dxv(R_ST2)) / dlx - (dyv(R_ST1)) / dly;
      stiff_source(I.sigma, W, vx, vy, vz, Ex, Ey, Ez, Bx, By, Bz, K[K_SEX], K[K_SEY], K[K_SEZ]);

      if (sa.mode == 1) {
#pragma unroll
        for (int c = 0; c < NRHS; ++c) I.rhs_out[c * fs + pc] = K[c];
      } else {
        // sumfin, 18_sumfin.f95:20-66
        double fin[NCONS];
#pragma unroll
        for (int c = 0; c < NCONS; ++c) {
          const double prev = (sa.l == 1) ? 0.0 : I.finsum[c * fs + pc];
          if (c >= Q_EX && c <= Q_EZ) fin[c] = prev + (sa.wb * K[c] - sa.wbt * K[K_SEX + (c - Q_EX)]);
          else fin[c] = prev + sa.wb * K[c];
        }
        // time-n conserved state U^n (prims for psi, phi, E, B, q; startconvar for D, tau, S)
        double U[NCONS];
        U[Q_PSI] = prim[P_PSI * fs + pc]; U[Q_PHI] = prim[P_PHI * fs + pc];
        U[Q_EX] = prim[P_EX * fs + pc]; U[Q_EY] = prim[P_EY * fs + pc]; U[Q_EZ] = prim[P_EZ * fs + pc];
        U[Q_BX] = prim[P_BX * fs + pc]; U[Q_BY] = prim[P_BY * fs + pc]; U[Q_BZ] = prim[P_BZ * fs + pc];
        U[Q_Q] = prim[P_Q * fs + pc];
        U[Q_D] = aux[A_D * fs + pc]; U[Q_TAU] = aux[A_TAU * fs + pc];
        U[Q_SX] = aux[A_SX * fs + pc]; U[Q_SY] = aux[A_SY * fs + pc]; U[Q_SZ] = aux[A_SZ * fs + pc];
        if (sa.l < sa.s) {
#pragma unroll
          for (int c = 0; c < NCONS; ++c) I.finsum[c * fs + pc] = fin[c];
          // sumint for stage l+1 (09_sumint.f95:18-67); intsum is zeroed only
          // once per step (07_clean_var.f95), so it accumulates across stages
          double acc[NCONS];
#pragma unroll
          for (int c = 0; c < NCONS; ++c) acc[c] = sa.need_intsum_load ? I.intsum[c * fs + pc] : 0.0;
          for (int m = 1; m <= sa.l; ++m) {
            const double ab = sa.ab_next[m - 1], abt = sa.abt_next[m - 1];
            if (ab == 0.0 && abt == 0.0) continue;
            const double* Km = (m < sa.l) ? I.kbuf + (long long)sa.kslot[m - 1] * NRHS * fs : nullptr;
#pragma unroll
            for (int c = 0; c < NCONS; ++c) {
              const double F = Km ? Km[c * fs + pc] : K[c];
              if (c >= Q_EX && c <= Q_EZ) {
                const double S = Km ? Km[(K_SEX + c - Q_EX) * fs + pc] : K[K_SEX + c - Q_EX];
                acc[c] = acc[c] + (ab * F - abt * S);
              } else {
                acc[c] = acc[c] + ab * F;
              }
            }
          }
          if (sa.need_intsum_store) {
#pragma unroll
            for (int c = 0; c < NCONS; ++c) I.intsum[c * fs + pc] = acc[c];
          }
          if (sa.store_k_slot >= 0) {
            double* Ko = I.kbuf + (long long)sa.store_k_slot * NRHS * fs;
#pragma unroll
            for (int c = 0; c < NRHS; ++c) Ko[c * fs + pc] = K[c];
          }
          // varint (10_varint.f95:23-63), electricvarint and flowinit of stage l+1
          double Qn[NCONS];
#pragma unroll
          for (int c = 0; c < NCONS; ++c) Qn[c] = U[c] + I.dt * acc[c];
          double Exn, Eyn, Ezn, Jx, Jy, Jz;
          implicit_e(sa.abt_diag_next, I.sigma, I.dt, W, vx, vy, vz, Qn[Q_BX], Qn[Q_BY], Qn[Q_BZ], Qn[Q_EX],
                     Qn[Q_EY], Qn[Q_EZ], Exn, Eyn, Ezn);
          Qn[Q_EX] = Exn; Qn[Q_EY] = Eyn; Qn[Q_EZ] = Ezn;
          current(I.sigma, W, vx, vy, vz, Exn, Eyn, Ezn, Qn[Q_BX], Qn[Q_BY], Qn[Q_BZ], Qn[Q_Q], Jx, Jy, Jz);
          double* Qo = I.stage[1 - sa.qin];
#pragma unroll
          for (int c = 0; c < NCONS; ++c) Qo[c * fs + pc] = Qn[c];
          Qo[Q_JX * fs + pc] = Jx; Qo[Q_JY * fs + pc] = Jy; Qo[Q_JZ * fs + pc] = Jz;
        } else {
          // varfin + electricfield (19_varfin.f95:39-51, 20_electricfield.f95:157-161)
          double Un[NCONS];
#pragma unroll
          for (int c = 0; c < NCONS; ++c) Un[c] = U[c] + I.dt * fin[c];
          // con2prim, l_swap = 1 (main_cueva_code.f95:312-326)
          C2PIn in{Un[Q_D], Un[Q_TAU], Un[Q_SX], Un[Q_SY], Un[Q_SZ], Un[Q_EX], Un[Q_EY], Un[Q_EZ],
                   Un[Q_BX], Un[Q_BY], Un[Q_BZ], vx, vy, vz, prim[P_RHO * fs + pc], prim[P_P * fs + pc]};
          C2POut o;
          st |= c2p_dispatch(I, in, o);
          double pv[NPRIM];
          pv[P_RHO] = o.rho; pv[P_P] = o.p; pv[P_VX] = o.vx; pv[P_VY] = o.vy; pv[P_VZ] = o.vz;
          pv[P_PSI] = Un[Q_PSI]; pv[P_PHI] = Un[Q_PHI];
          pv[P_EX] = Un[Q_EX]; pv[P_EY] = Un[Q_EY]; pv[P_EZ] = Un[Q_EZ];
          pv[P_BX] = Un[Q_BX]; pv[P_BY] = Un[Q_BY]; pv[P_BZ] = Un[Q_BZ]; pv[P_Q] = Un[Q_Q];
          double* po = I.prim[1 - sa.cur];
#pragma unroll
          for (int c = 0; c < NPRIM; ++c) po[c * fs + pc] = pv[c];
          begin_step_point(I, sa.abt_diag_first, I.aux[1 - sa.cur], I.stage[1 - sa.qin], pc, pv);
        }
      }
    }
    if (st) atomicOr(I.status, st);
#pragma unroll
    for (int c = 0; c < NROLE; ++c) prevFy[c] = Fy[c];
  }
}

// ---------------------------------------------------------------- launchers
template <int RM, int SV>
static cudaError_t launch_rm_sv(int prec, int nblocks, cudaStream_t st, const InstDesc* d, int n, const StageArgs& sa) {
  if (prec == 0) k_sweep<RM, SV, double><<<nblocks, SWEEP_WARPS * 32, 0, st>>>(d, n, sa);
  else k_sweep<RM, SV, float><<<nblocks, SWEEP_WARPS * 32, 0, st>>>(d, n, sa);
  return cudaGetLastError();
}

cudaError_t launch_sweep(int rec_mp, int solver, int prec, int nblocks, cudaStream_t st, const InstDesc* d, int n,
                         const StageArgs& sa) {
  if (nblocks <= 0) return cudaSuccess;
  switch (rec_mp * 10 + (solver == 7 ? 1 : 0)) {
    case 0: return launch_rm_sv<0, 5>(prec, nblocks, st, d, n, sa);
    case 1: return launch_rm_sv<0, 7>(prec, nblocks, st, d, n, sa);
    case 10: return launch_rm_sv<1, 5>(prec, nblocks, st, d, n, sa);
    case 11: return launch_rm_sv<1, 7>(prec, nblocks, st, d, n, sa);
    case 20: return launch_rm_sv<2, 5>(prec, nblocks, st, d, n, sa);
    case 21: return launch_rm_sv<2, 7>(prec, nblocks, st, d, n, sa);
    default: return cudaErrorInvalidValue;
  }
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
cudaError_t launch_con2prim(long long npts, cudaStream_t st, const InstDesc* d, int n, int cur) {
  k_con2prim<<<point_grid(npts, n), 256, 0, st>>>(d, cur);
  return cudaGetLastError();
}

}  // namespace cueva
