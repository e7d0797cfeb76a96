// cueva_kernels.cu -- sm_100a kernels of the CUEVA per-step hot path.
//
// One RK stage = three launches:
//  k_face<..., 0>  one thread per x interface (i+1/2, j), stencils staged
//                  in shared memory: MP5/7/9 reconstruction of the 21 x
//                  slots plus the y velocities (and y densities for HLLC)
//                  at (i, j) that the reference's fix-ups couple in, then
//                  the HLL / HLLC flux; 14 fluxes written to a scratch slab;
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
// A CTA covers 32 interfaces along the row times FACE_ROWS rows.  Every
// value its stencils read is first copied into shared memory with cp.async
// (all copies in flight at once, one wait), so the reconstruction and the
// Riemann solve run from shared memory without global-load latency.
//   x faces (D = 0): i = i0-1+lane in [-1, imax], j = j0+warp in [0, jmax];
//   y faces (D = 1): i = i0+lane in [0, imax], j = j0-1+warp in [-1, jmax]
// (the interfaces 17_fluxandsource.f95 differences).  Staged regions:
//   normal:     NF fields x FACE_ROWS rows x (32 + 2R + 1) cells along the
//               normal (x) or NF fields x (FACE_ROWS + 2R + 1) rows x 32
//               columns (y);
//   transverse: the NC velocity (+ density) fields the fix-ups couple in,
//               along the other direction through the face's cell.
__device__ __forceinline__ void cp_async8(double* sdst, const double* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

constexpr int NF_FACE = 20;   // 5 primitive slots + 14 conserved + the normal current

template <int RM, int SOLVER>
struct FaceGeom {
  static constexpr int R = MPR<RM>::R;
  static constexpr int NS = 2 * R + 2;                 // stencil points
  static constexpr int LONG = 32 + 2 * R + 1;          // staged cells along a 32-face segment
  static constexpr int DEEP = FACE_ROWS + 2 * R + 1;   // staged rows across FACE_ROWS faces
  static constexpr int NC = (SOLVER == 7) ? 4 : 3;     // coupled fields: v (+ rho for HLLC)
  // D = 0: normal [row][f][LONG], transverse [f][DEEP][32]
  // D = 1: normal [f][DEEP][32],  transverse [row][f][LONG]
  static constexpr int NORMAL0 = FACE_ROWS * NF_FACE * LONG;
  static constexpr int NORMAL1 = NF_FACE * DEEP * 32;
  static constexpr int TRANS0 = NC * DEEP * 32;
  static constexpr int TRANS1 = FACE_ROWS * NC * LONG;
  static constexpr size_t bytes(int D) {
    return sizeof(double) * (size_t)(D == 0 ? NORMAL0 + TRANS0 : NORMAL1 + TRANS1);
  }
};

template <int RM, int SOLVER, typename T, int D>
__global__ void __launch_bounds__(32 * FACE_ROWS, 2)
k_face(const InstDesc* __restrict__ insts, int ninst, StageArgs sa) {
  using G = FaceGeom<RM, SOLVER>;
  constexpr int R = G::R, NS = G::NS, LONG = G::LONG, DEEP = G::DEEP, NC = G::NC;
  extern __shared__ double smem[];
  int b = blockIdx.x, k = 0;
  for (int t = 1; t < ninst; ++t)
    if (insts[t].block_begin[D] <= b) k = t;
  const InstDesc& I = insts[k];
  b -= I.block_begin[D];
  const int imax = I.imax, jmax = I.jmax, pitch = I.pitch, bcx = I.bc_x, bcy = I.bc_y;
  const int lane = threadIdx.x, w = threadIdx.y, tid = w * 32 + lane;
  const int nfr = (D == 0) ? imax + 2 : imax + 1;      // faces per row
  const int bpr = (nfr + 31) / 32;
  const int i0 = (b % bpr) * 32 - (D == 0 ? 1 : 0);      // first face of the segment
  const int j0 = (b / bpr) * FACE_ROWS - (D == 1 ? 1 : 0);
  const int i = i0 + lane, j = j0 + w;
  const long long fs = I.fstride;
  const double* __restrict__ prim = I.prim[sa.cur];
  const double* __restrict__ Q = I.stage[sa.qin];
  // staged field f: 0-4 primitive slots (vx, vy, vz, p, rho), 5-19 stage
  // fields psi..Sz and the current along the normal
  auto field = [&](int f) -> const double* {
    if (f < 5) {
      const int pf = (f < 3) ? P_VX + f : (f == 3 ? P_P : P_RHO);
      return prim + (long long)pf * fs;
    }
    const int qf = (f < 19) ? f - 5 : (D == 0 ? Q_JX : Q_JY);
    return Q + (long long)qf * fs;
  };
  // coupled field c: vx, vy, vz, rho
  auto cfield = [&](int c) -> const double* { return prim + (long long)(c < 3 ? P_VX + c : P_RHO) * fs; };
  double* sn = smem;
  double* st = smem + (D == 0 ? G::NORMAL0 : G::NORMAL1);
  const int ilast = min(i0 + 31, imax), jlast = min(j0 + FACE_ROWS - 1, jmax);  // last face of the tile

  // ---- stage the stencils (cells reaching beyond the last face are skipped)
  if constexpr (D == 0) {
    // normal: rows j0..jlast, cells i0-R .. ilast+R+1 along x
    const int ncell = ilast + R + 1 - (i0 - R) + 1;
    for (int e = tid; e < FACE_ROWS * LONG; e += 32 * FACE_ROWS) {
      const int r = e / LONG, c = e - r * LONG;
      if (j0 + r > jlast || c >= ncell) continue;
      const long long off = (long long)map_idx(j0 + r, jmax, bcy) * pitch + map_idx(i0 - R + c, imax, bcx);
      double* d = sn + (r * NF_FACE) * LONG + c;
#pragma unroll
      for (int f = 0; f < NF_FACE; ++f) cp_async8(d + f * LONG, field(f) + off);
    }
    // transverse: columns i0..ilast, rows j0-R .. jlast+R+1 along y
    const int nrow = jlast + R + 1 - (j0 - R) + 1;
    for (int e = tid; e < DEEP * 32; e += 32 * FACE_ROWS) {
      const int r = e >> 5, c = e & 31;
      if (r >= nrow || i0 + c > ilast) continue;
      const long long off = (long long)map_idx(j0 - R + r, jmax, bcy) * pitch + map_idx(i0 + c, imax, bcx);
#pragma unroll
      for (int f = 0; f < NC; ++f) cp_async8(st + (f * DEEP + r) * 32 + c, cfield(f) + off);
    }
  } else {
    // normal: columns i0..ilast, rows j0-R .. jlast+R+1 along y
    const int nrow = jlast + R + 1 - (j0 - R) + 1;
    for (int e = tid; e < DEEP * 32; e += 32 * FACE_ROWS) {
      const int r = e >> 5, c = e & 31;
      if (r >= nrow || i0 + c > ilast) continue;
      const long long off = (long long)map_idx(j0 - R + r, jmax, bcy) * pitch + map_idx(i0 + c, imax, bcx);
#pragma unroll
      for (int f = 0; f < NF_FACE; ++f) cp_async8(sn + (f * DEEP + r) * 32 + c, field(f) + off);
    }
    // transverse: rows j0..jlast, cells i0-R .. ilast+R+1 along x
    const int ncell = ilast + R + 1 - (i0 - R) + 1;
    for (int e = tid; e < FACE_ROWS * LONG; e += 32 * FACE_ROWS) {
      const int r = e / LONG, c = e - r * LONG;
      if (j0 + r > jlast || c >= ncell) continue;
      const long long off = (long long)map_idx(j0 + r, jmax, bcy) * pitch + map_idx(i0 - R + c, imax, bcx);
#pragma unroll
      for (int f = 0; f < NC; ++f) cp_async8(st + (r * NC + f) * LONG + c, cfield(f) + off);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  if (i > ilast || j > jlast) return;

  // stencil of staged field f through this face (normal) / the face's cell (transverse)
  auto nrmd = [&](int f, int q) -> double {
    return (D == 0) ? sn[(w * NF_FACE + f) * LONG + lane + q] : sn[(f * DEEP + w + q) * 32 + lane];
  };
  auto nrm = [&](int f, int q) -> T { return T(nrmd(f, q)); };
  auto trn = [&](int f, int q) -> T {
    return (D == 0) ? T(st[(f * DEEP + w + q) * 32 + lane]) : T(st[(w * NC + f) * LONG + lane + q]);
  };
  auto rec = [&](int f, T& L, T& Rv) {
    T u[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) u[q] = nrm(f, q);
    const Pair<T> p = MPCall<RM, T>::template call<false>(u);
    L = p.L; Rv = p.R;
  };
  auto recp = [&](int f, T& L, T& Rv) {
    T u[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) u[q] = nrm(f, q);
    const Pair<T> p = MPCall<RM, T>::template call<true>(u);
    L = p.L; Rv = p.R;
  };
  auto rect = [&](int f, bool pos, T& L, T& Rv) {
    T u[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) u[q] = trn(f, q);
    const Pair<T> p = pos ? MPCall<RM, T>::template call<true>(u) : MPCall<RM, T>::template call<false>(u);
    L = p.L; Rv = p.R;
  };

  uint32_t stt = 0;
  Side<T> L, Rs;
  // primitive slots of this direction (21-25 for x, 58-62 for y)
  rec(0, L.vx, Rs.vx);
  rec(1, L.vy, Rs.vy);
  rec(2, L.vz, Rs.vz);
  recp(3, L.p, Rs.p);
  recp(4, L.rho, Rs.rho);
  if constexpr (SOLVER == 5 || SOLVER == 7) {
    // superluminal fall-back, 16_hll_flow_mpx.f95:1393-1462: the x and y
    // reconstructions of the point fall back together if either is
    // superluminal; left states take cell (i,j), right states cell i-1 (x)
    // or j-1 (y), as in the reference
    T ovx, ovy, ovz, wvx, wvy, wvz;
    rect(0, false, ovx, wvx);
    rect(1, false, ovy, wvy);
    rect(2, false, ovz, wvz);
    const T V2l = pw2(L.vx) + pw2(L.vy) + pw2(L.vz);
    const T V2r = pw2(Rs.vx) + pw2(Rs.vy) + pw2(Rs.vz);
    const T V2ol = pw2(ovx) + pw2(ovy) + pw2(ovz);
    const T V2or = pw2(wvx) + pw2(wvy) + pw2(wvz);
    if (V2l >= T(1) || V2r >= T(1) || V2ol >= T(1) || V2or >= T(1)) {
      // cell (i, j) is stencil point R of the normal stencil; i-1 / j-1 is R-1
      L.vx = nrm(0, R); L.vy = nrm(1, R); L.vz = nrm(2, R);
      Rs.vx = nrm(0, R - 1); Rs.vy = nrm(1, R - 1); Rs.vz = nrm(2, R - 1);
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
        rect(3, true, oL, oR);
        other_neg = (oL < T(0)) || (oR < T(0));
      }
      if (!other_neg) {
        const T r10 = T(nrmd(4, R) * 1.0e-1);
        if (L.rho < T(0)) L.rho = r10;
        else Rs.rho = r10;
      }
    }
  }
  rec(5 + Q_PSI, L.psi, Rs.psi);
  rec(5 + Q_PHI, L.phi, Rs.phi);
  rec(5 + Q_EX, L.Ex, Rs.Ex);
  rec(5 + Q_EY, L.Ey, Rs.Ey);
  rec(5 + Q_EZ, L.Ez, Rs.Ez);
  rec(5 + Q_BX, L.Bx, Rs.Bx);
  rec(5 + Q_BY, L.By, Rs.By);
  rec(5 + Q_BZ, L.Bz, Rs.Bz);
  rec(5 + Q_Q, L.q, Rs.q);
  rec(5 + Q_D, L.D, Rs.D);
  rec(5 + Q_TAU, L.tau, Rs.tau);
  rec(5 + Q_SX, L.Sx, Rs.Sx);
  rec(5 + Q_SY, L.Sy, Rs.Sy);
  rec(5 + Q_SZ, L.Sz, Rs.Sz);
  rec(19, L.J, Rs.J);
  const T gamma = T(I.gamma);
  T F[NROLE];
  if constexpr (SOLVER == 5) hll_fluxes<D>(L, Rs, gamma, F);
  else hllc_fluxes<D>(L, Rs, gamma, F, stt);
  double* out = (D == 0) ? I.fx : I.fy;
  const long long fo = (D == 0) ? (long long)j * I.fpitch + (i + 1) : (long long)(j + 1) * I.fpitch + i;
#pragma unroll
  for (int c = 0; c < NROLE; ++c) out[c * I.ffs + fo] = double(F[c]);
  if (stt) atomicOr(I.status, stt);
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
  const double dlx = I.delx, dly = I.dely, ix2 = I.inv_delx_pow2, iy2 = I.inv_dely_pow2;
  auto dxq = [&](int r) { return ix2 != 0.0 ? dxv(r) * ix2 : dxv(r) / dlx; };   // (dx)/dlx
  auto dyq = [&](int r) { return iy2 != 0.0 ? dyv(r) * iy2 : dyv(r) / dly; };   // (dy)/dly
  // centre values of stage l and time n
  const double q = Q[Q_Q * fs + pc], psi = Q[Q_PSI * fs + pc], phi = Q[Q_PHI * fs + pc];
  const double Ex = Q[Q_EX * fs + pc], Ey = Q[Q_EY * fs + pc], Ez = Q[Q_EZ * fs + pc];
  const double Bx = Q[Q_BX * fs + pc], By = Q[Q_BY * fs + pc], Bz = Q[Q_BZ * fs + pc];
  const double vx = prim[P_VX * fs + pc], vy = prim[P_VY * fs + pc], vz = prim[P_VZ * fs + pc];
  const double W = aux[A_W * fs + pc];
  double K[NRHS];
  // 17_fluxandsource.f95:488-598; z differences are (X - X)/Delz = 0
  // (-a)/d == -(a/d) exactly, so every term is -/+ the quotient of a difference
  K[Q_PSI] = -dxq(R_PSI) - dyq(R_PSI) + q - I.kappa_psi * psi;
  K[Q_PHI] = -dxq(R_PHI) - dyq(R_PHI) - I.kappa_phi * phi;
  K[Q_BX] = -dyq(R_BT2) + 0.0 - dxq(R_BN);
  K[Q_BY] = dxq(R_BT1) - dyq(R_BN);
  K[Q_BZ] = -dxq(R_BT2) + dyq(R_BT1);
  K[Q_EX] = dyq(R_ET2) - dxq(R_EN) - q * vx;
  K[Q_EY] = 0.0 - dxq(R_ET1) - dyq(R_EN) - q * vy;
  K[Q_EZ] = dxq(R_ET2) - dyq(R_ET1) - q * vz;
  K[Q_Q] = -dxq(R_Q) - dyq(R_Q);
  K[Q_D] = -dxq(R_D) - dyq(R_D);
  K[Q_TAU] = -dxq(R_TAU) - dyq(R_TAU);
  K[Q_SX] = -dxq(R_SN) - dyq(R_ST2);
  K[Q_SY] = -dxq(R_ST1) - dyq(R_SN);
  K[Q_SZ] = -dxq(R_ST2) - dyq(R_ST1);
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
  using G = FaceGeom<RM, SV>;
  const dim3 blk(32, FACE_ROWS);
  if (ev) cudaEventRecord(ev[0], st);
  k_face<RM, SV, T, 0><<<nb[LK_XFACE], blk, G::bytes(0), st>>>(d, n, sa);
  if (ev) cudaEventRecord(ev[1], st);
  k_face<RM, SV, T, 1><<<nb[LK_YFACE], blk, G::bytes(1), st>>>(d, n, sa);
  if (ev) cudaEventRecord(ev[2], st);
}

template <int RM, int SV, typename T>
static cudaError_t prepare_faces() {
  using G = FaceGeom<RM, SV>;
  cudaError_t e = cudaFuncSetAttribute(k_face<RM, SV, T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)G::bytes(0));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_face<RM, SV, T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::bytes(1));
  return e;
}

template <int RM, int SV>
static cudaError_t prepare_rm_sv(int prec) {
  return prec == 0 ? prepare_faces<RM, SV, double>() : prepare_faces<RM, SV, float>();
}

cudaError_t prepare_stage(int rec_mp, int solver, int prec) {
  switch (rec_mp * 10 + (solver == 7 ? 1 : 0)) {
    case 0: return prepare_rm_sv<0, 5>(prec);
    case 1: return prepare_rm_sv<0, 7>(prec);
    case 10: return prepare_rm_sv<1, 5>(prec);
    case 11: return prepare_rm_sv<1, 7>(prec);
    case 20: return prepare_rm_sv<2, 5>(prec);
    case 21: return prepare_rm_sv<2, 7>(prec);
    default: return cudaErrorInvalidValue;
  }
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
