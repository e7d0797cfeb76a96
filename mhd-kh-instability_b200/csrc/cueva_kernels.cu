// cueva_kernels.cu -- sm_100a kernels of the CUEVA per-step hot path.
//
// One RK stage = three launches:
//  k_face<..., 0>  one thread per x interface (i+1/2, j): MP5/7/9
//                  reconstruction of the 21 x slots plus the y velocities
//                  (and y densities for HLLC) at (i, j) that the reference's
//                  fix-ups couple in, then the HLL / HLLC flux; 14 fluxes
//                  written to a scratch slab;
//  k_face<..., 1>  the same for the y interfaces (i, j+1/2);
//  k_update<EP>    one thread per grid point: flux divergence and sources
//                  (17_fluxandsource.f95:441-635) and a fused pointwise
//                  epilogue -- sumfin, the next stage's sumint / varint /
//                  electricvarint / flowinit, or, after the last stage,
//                  varfin / electricfield, con2prim and the next step's
//                  startconvar.
// The reference computes both faces of a point in one loop iteration
// (16_hll_flow_mpx.f95:1358-1965); splitting them keeps one direction's
// state per thread (register pressure, occupancy) at the cost of the
// 28-double flux round trip through L2/HBM.
#include <cuda_runtime.h>
#include <math_constants.h>

#include "cueva_common.cuh"
#include "cueva_mp.cuh"
#include "cueva_riemann.cuh"
#include "cueva_point.cuh"
#include "cueva_mlp.cuh"

namespace cueva {

// ------------------------------------------------------------------ helpers
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

// ------------------------------------------------------------ face kernels
// x faces: i in [-1, imax], j in [0, jmax]; y faces: i in [0, imax],
// j in [-1, jmax] (the interfaces 17_fluxandsource.f95 differences)
template <int RM, int SOLVER, typename T, int D>
__global__ void __launch_bounds__(32 * FACE_ROWS)
k_face(const InstDesc* __restrict__ insts, int ninst, StageArgs sa) {
  constexpr int R = MPR<RM>::R;
  constexpr int NS = 2 * R + 2;
  int b = blockIdx.x, k = 0;
  for (int t = 1; t < ninst; ++t)
    if (insts[t].block_begin[D] <= b) k = t;
  const InstDesc& I = insts[k];
  b -= I.block_begin[D];
  const int imax = I.imax, jmax = I.jmax, pitch = I.pitch, bcx = I.bc_x, bcy = I.bc_y;
  const int nfx = (D == 0) ? imax + 2 : imax + 1;          // faces per row
  const int bpr = (nfx + 31) / 32;
  const int i = (b % bpr) * 32 + (int)threadIdx.x - (D == 0 ? 1 : 0);
  const int j = (b / bpr) * FACE_ROWS + (int)threadIdx.y - (D == 1 ? 1 : 0);
  if (i > imax || j > jmax) return;
  const long long fs = I.fstride;
  const T gamma = T(I.gamma);
  const double* __restrict__ prim = I.prim[sa.cur];
  const double* __restrict__ Q = I.stage[sa.qin];

  // stencil offsets: along the normal (cells n-R .. n+1+R) and, for the
  // coupled fix-ups, along the other direction through the same point
  int offn[NS], offt[NS];
  const int ci = map_idx(i, imax, bcx), rj = map_idx(j, jmax, bcy);
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    if (D == 0) {
      offn[q] = rj * pitch + map_idx(i - R + q, imax, bcx);
      offt[q] = map_idx(j - R + q, jmax, bcy) * pitch + ci;
    } else {
      offn[q] = map_idx(j - R + q, jmax, bcy) * pitch + ci;
      offt[q] = rj * pitch + map_idx(i - R + q, imax, bcx);
    }
  }
  auto rec = [&](const double* f, const int (&off)[NS], T& L, T& Rv) {
    T u[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) u[q] = ldT<T>(f + off[q]);
    const Pair<T> p = MPCall<RM, T>::template call<false>(u);
    L = p.L; Rv = p.R;
  };
  auto recp = [&](const double* f, const int (&off)[NS], T& L, T& Rv) {
    T u[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) u[q] = ldT<T>(f + off[q]);
    const Pair<T> p = MPCall<RM, T>::template call<true>(u);
    L = p.L; Rv = p.R;
  };

  uint32_t st = 0;
  Side<T> L, Rs;
  // primitive slots of this direction (21-25 for x, 58-62 for y)
  rec(prim + P_VX * fs, offn, L.vx, Rs.vx);
  rec(prim + P_VY * fs, offn, L.vy, Rs.vy);
  rec(prim + P_VZ * fs, offn, L.vz, Rs.vz);
  recp(prim + P_P * fs, offn, L.p, Rs.p);
  recp(prim + P_RHO * fs, offn, L.rho, Rs.rho);
  if constexpr (SOLVER == 5 || SOLVER == 7) {
    // superluminal fall-back, 16_hll_flow_mpx.f95:1393-1462: the x and y
    // reconstructions of the point fall back together if either is
    // superluminal; left states take cell (i,j), right states cell i-1 (x)
    // or j-1 (y), as in the reference
    T ovx, ovy, ovz, wvx, wvy, wvz;
    rec(prim + P_VX * fs, offt, ovx, wvx);
    rec(prim + P_VY * fs, offt, ovy, wvy);
    rec(prim + P_VZ * fs, offt, ovz, wvz);
    const T V2l = pw2(L.vx) + pw2(L.vy) + pw2(L.vz);
    const T V2r = pw2(Rs.vx) + pw2(Rs.vy) + pw2(Rs.vz);
    const T V2ol = pw2(ovx) + pw2(ovy) + pw2(ovz);
    const T V2or = pw2(wvx) + pw2(wvy) + pw2(wvz);
    if (V2l >= T(1) || V2r >= T(1) || V2ol >= T(1) || V2or >= T(1)) {
      const int c0 = rj * pitch + ci;
      const int cm = (D == 0) ? rj * pitch + map_idx(i - 1, imax, bcx) : map_idx(j - 1, jmax, bcy) * pitch + ci;
      L.vx = ldT<T>(prim + P_VX * fs + c0); L.vy = ldT<T>(prim + P_VY * fs + c0); L.vz = ldT<T>(prim + P_VZ * fs + c0);
      Rs.vx = ldT<T>(prim + P_VX * fs + cm); Rs.vy = ldT<T>(prim + P_VY * fs + cm); Rs.vz = ldT<T>(prim + P_VZ * fs + cm);
    }
  }
  if constexpr (SOLVER == 7) {
    // density fix-up chain, 16_hllc_flow_mpx.f95:2663-2690: the first
    // negative of (yL, yR, xL, xR) becomes 0.1 rho(i,j); an x side is only
    // fixed when neither y side is negative
    if (L.rho < T(0) || Rs.rho < T(0)) {
      bool other_neg = false;
      if (D == 0) {
        T oL, oR;
        recp(prim + P_RHO * fs, offt, oL, oR);
        other_neg = (oL < T(0)) || (oR < T(0));
      }
      if (!other_neg) {
        const T r10 = T(__ldg(prim + P_RHO * fs + rj * pitch + ci) * 1.0e-1);
        if (L.rho < T(0)) L.rho = r10;
        else Rs.rho = r10;
      }
    }
  }
  rec(Q + Q_PSI * fs, offn, L.psi, Rs.psi);
  rec(Q + Q_PHI * fs, offn, L.phi, Rs.phi);
  rec(Q + Q_EX * fs, offn, L.Ex, Rs.Ex);
  rec(Q + Q_EY * fs, offn, L.Ey, Rs.Ey);
  rec(Q + Q_EZ * fs, offn, L.Ez, Rs.Ez);
  rec(Q + Q_BX * fs, offn, L.Bx, Rs.Bx);
  rec(Q + Q_BY * fs, offn, L.By, Rs.By);
  rec(Q + Q_BZ * fs, offn, L.Bz, Rs.Bz);
  rec(Q + Q_Q * fs, offn, L.q, Rs.q);
  rec(Q + Q_D * fs, offn, L.D, Rs.D);
  rec(Q + Q_TAU * fs, offn, L.tau, Rs.tau);
  rec(Q + Q_SX * fs, offn, L.Sx, Rs.Sx);
  rec(Q + Q_SY * fs, offn, L.Sy, Rs.Sy);
  rec(Q + Q_SZ * fs, offn, L.Sz, Rs.Sz);
  rec(Q + (D == 0 ? Q_JX : Q_JY) * fs, offn, L.J, Rs.J);
  T F[NROLE];
  if constexpr (SOLVER == 5) hll_fluxes<D>(L, Rs, gamma, F);
  else hllc_fluxes<D>(L, Rs, gamma, F, st);
  double* out = (D == 0) ? I.fx : I.fy;
  const long long fo = (D == 0) ? (long long)j * I.fpitch + (i + 1) : (long long)(j + 1) * I.fpitch + i;
#pragma unroll
  for (int c = 0; c < NROLE; ++c) out[c * I.ffs + fo] = double(F[c]);
  if (st) atomicOr(I.status, st);
}

// ------------------------------------------------------------ update kernel
// EP selects the epilogue: EP_RHS stores the stage right-hand side only (the
// routine mirror), EP_MID prepares stage l+1, EP_LAST finishes the step.
enum Epilogue { EP_RHS = 0, EP_MID = 1, EP_LAST = 2 };

template <int EP>
__global__ void __launch_bounds__(POINT_THREADS)
k_update(const InstDesc* __restrict__ insts, int ninst, StageArgs sa) {
  int b = blockIdx.x, k = 0;
  for (int t = 1; t < ninst; ++t)
    if (insts[t].block_begin[LK_POINT] <= b) k = t;
  const InstDesc& I = insts[k];
  b -= I.block_begin[LK_POINT];
  const int nx = I.imax + 1;
  const int bpr = (nx + 31) / 32;
  const int i = (b % bpr) * 32 + (int)(threadIdx.x & 31);
  const int j = (b / bpr) * (POINT_THREADS / 32) + (int)(threadIdx.x >> 5);
  if (i > I.imax || j > I.jmax) return;
  const int pitch = I.pitch;
  const long long fs = I.fstride;
  const double* __restrict__ prim = I.prim[sa.cur];
  const double* __restrict__ aux = I.aux[sa.cur];
  const double* __restrict__ Q = I.stage[sa.qin];
  uint32_t st = 0;
  const long long pc = (long long)j * pitch + i;
  const long long fxo = (long long)j * I.fpitch + (i + 1);      // Fx(i+1/2, j); Fx(i-1/2, j) at -1
  const long long fyo = (long long)(j + 1) * I.fpitch + i;      // Fy(i, j+1/2); Fy(i, j-1/2) at -fpitch
  const double* __restrict__ fx = I.fx;
  const double* __restrict__ fy = I.fy;
  auto dxv = [&](int r) { return fx[r * I.ffs + fxo] - fx[r * I.ffs + fxo - 1]; };
  auto dyv = [&](int r) { return fy[r * I.ffs + fyo] - fy[r * I.ffs + fyo - I.fpitch]; };
  const double dlx = I.delx, dly = I.dely;
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

  if constexpr (EP == EP_RHS) {
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
    if constexpr (EP == EP_MID) {
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
  if (st) atomicOr(I.status, st);
}

// ---------------------------------------------------------------- launchers
template <int RM, int SV, typename T>
static void launch_faces(const int (&nb)[3], cudaStream_t st, const InstDesc* d, int n, const StageArgs& sa,
                         cudaEvent_t* ev) {
  const dim3 blk(32, FACE_ROWS);
  if (ev) cudaEventRecord(ev[0], st);
  k_face<RM, SV, T, 0><<<nb[LK_XFACE], blk, 0, st>>>(d, n, sa);
  if (ev) cudaEventRecord(ev[1], st);
  k_face<RM, SV, T, 1><<<nb[LK_YFACE], blk, 0, st>>>(d, n, sa);
  if (ev) cudaEventRecord(ev[2], st);
}

template <int RM, int SV>
static void launch_rm_sv(int prec, const int (&nb)[3], cudaStream_t st, const InstDesc* d, int n,
                         const StageArgs& sa, cudaEvent_t* ev) {
  if (prec == 0) launch_faces<RM, SV, double>(nb, st, d, n, sa, ev);
  else launch_faces<RM, SV, float>(nb, st, d, n, sa, ev);
}

cudaError_t launch_stage(int rec_mp, int solver, int prec, const int (&nb)[3], cudaStream_t st, const InstDesc* d,
                         int n, const StageArgs& sa, cudaEvent_t* ev) {
  switch (rec_mp * 10 + (solver == 7 ? 1 : 0)) {
    case 0: launch_rm_sv<0, 5>(prec, nb, st, d, n, sa, ev); break;
    case 1: launch_rm_sv<0, 7>(prec, nb, st, d, n, sa, ev); break;
    case 10: launch_rm_sv<1, 5>(prec, nb, st, d, n, sa, ev); break;
    case 11: launch_rm_sv<1, 7>(prec, nb, st, d, n, sa, ev); break;
    case 20: launch_rm_sv<2, 5>(prec, nb, st, d, n, sa, ev); break;
    case 21: launch_rm_sv<2, 7>(prec, nb, st, d, n, sa, ev); break;
    default: return cudaErrorInvalidValue;
  }
  if (sa.mode == 1) k_update<EP_RHS><<<nb[LK_POINT], POINT_THREADS, 0, st>>>(d, n, sa);
  else if (sa.l < sa.s) k_update<EP_MID><<<nb[LK_POINT], POINT_THREADS, 0, st>>>(d, n, sa);
  else k_update<EP_LAST><<<nb[LK_POINT], POINT_THREADS, 0, st>>>(d, n, sa);
  if (ev) cudaEventRecord(ev[3], st);
  return cudaGetLastError();
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
