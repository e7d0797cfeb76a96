// cueva_stage.cuh -- the two stage kernels of the CUEVA hot path (templates),
// shared by the per-solver translation units cueva_stage_{lax,mcl,hllemc,hllcmc,hll,hllc,hlle}.cu
// and by the pointwise kernels of cueva_kernels.cu.
//
// One RK stage = two launches:
//  k_yface  one thread per y interface (i, j+1/2), stencils staged in shared
//           memory: MP5/7/9 reconstruction of the 20 y slots plus the x
//           velocities at (i, j) that the reference's superluminal fix-up
//           couples in, then the HLL / HLLC / HLLE flux; 14 fluxes to a
//           scratch slab;
//  k_xupd   one thread per x interface (i+1/2, j), same staging, plus the
//           y densities for the HLLC density fix-up chain; the x flux of the
//           neighbour interface arrives by warp shuffle, so each thread then
//           updates its point: flux divergence and sources
//           (17_fluxandsource.f95:441-635) and a fused pointwise epilogue --
//           sumfin, the next stage's sumint / varint / electricvarint /
//           flowinit, or, after the last stage, varfin / electricfield,
//           con2prim and the next step's startconvar.
// The reference computes both faces of a point in one loop iteration
// (16_hll_flow_mpx.f95:1358-1965); splitting the directions keeps one
// direction's state per thread (register pressure, occupancy) at the cost of
// the 14-double y-flux round trip through L2/HBM.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>

#include <type_traits>

#include "cueva_common.cuh"
#include "cueva_mp.cuh"
#include "cueva_riemann.cuh"
#include "cueva_point.cuh"
#include "cueva_mlp.cuh"
#include "cueva_umma.cuh"

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

// The reference lets NaN states pass silently (its comparisons are false on
// NaN); a non-finite recovered state is reported as ST_NONFINITE here.
// count == false: a lane that only keeps its warp converged (no counters);
// full_warp: all 32 lanes of the warp make this call
__device__ __forceinline__ uint32_t c2p_dispatch(const InstDesc& I, const C2PIn& in, C2POut& o, bool count = true,
                                                 bool full_warp = false) {
  uint32_t st;
  if (I.c2p == 1) st = c2p_cardano(in, I.gamma, I.eps1_c2p, o, count ? I.counters : nullptr);
  else if (I.c2p == 0) st = c2p_nr(in, I.gamma, o);
  else st = c2p_learned(in, I.gamma, I.eps1_c2p, I.mlp, o, I.counters, count, full_warp);
  if (!(isfinite(o.rho) && isfinite(o.p) && isfinite(o.vx) && isfinite(o.vy) && isfinite(o.vz))) st |= ST_NONFINITE;
  return st;
}

// ------------------------------------------------------------ face tiles
// A CTA covers 32 interfaces along the row times FACE_ROWS rows.  Every
// value its stencils read is first copied into shared memory with cp.async
// (all copies in flight at once, one wait), so the reconstruction and the
// Riemann solve run from shared memory without global-load latency.
//   x faces (D = 0): i = i0+lane, j = j0+warp;  y faces (D = 1): i = i0+lane,
//   j = j0+warp; face "i" is the interface i+1/2 (x) or j+1/2 (y).
// Staged regions:
//   normal:     NF_FACE fields x FACE_ROWS rows x (32 + 2R + 1) cells along
//               x (D = 0), or NF_FACE fields x (FACE_ROWS + 2R + 1) rows x 32
//               columns (D = 1);
//   transverse: the NC velocity (+ density) fields the fix-ups couple in,
//               along the other direction through the face's cell.
__device__ __forceinline__ void cp_async8(double* sdst, const double* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// L2 prefetch of the n doubles at p, widened to 16-byte boundaries (which
// stay inside the 256-byte-aligned row the doubles belong to)
template <typename E>
__device__ __forceinline__ void prefetch_l2(const E* p, int n) {
  const unsigned long long a = (unsigned long long)p & ~15ull;
  const unsigned long long e = ((unsigned long long)(p + n) + 15ull) & ~15ull;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(a), "r"((unsigned)(e - a)) : "memory");
}

// Type of the face fluxes a stage kernel produces: T, except that the
// mixed-precision MP solvers return FP64 (their field roles psi, phi, E, B
// are computed in FP64, the others are FP32 values held exactly).
template <typename T, int SV>
constexpr bool kEmF64 = sizeof(T) == 4 && mixed_em_f64(SV);
template <typename T, int SV>
using flux_t = typename std::conditional<kEmF64<T, SV>, double, T>::type;

// The y-flux scratch holds each flux in the type it is computed in (FP64,
// or FP32 for the mixed-precision kernels, the update converting it to FP64
// exactly as it would convert the register value), at the place flux_slot
// gives; element e of role c is element e of that slab.
template <typename T, int SV>
__device__ __forceinline__ void flux_store(double* fy, long long ffs, int c, long long e, double v) {
  const FluxSlot s = flux_slot(sizeof(T) == 4, SV, c, ffs);
  if (s.f64) fy[s.off + e] = v;
  else reinterpret_cast<float*>(fy)[s.off + e] = float(v);
}
template <typename T, int SV>
__device__ __forceinline__ double flux_load(const double* fy, long long ffs, int c, long long e) {
  const FluxSlot s = flux_slot(sizeof(T) == 4, SV, c, ffs);
  if (s.f64) return fy[s.off + e];
  return double(reinterpret_cast<const float*>(fy)[s.off + e]);
}
// L2 prefetch of n elements of role c from element e on
template <typename T, int SV>
__device__ __forceinline__ void flux_prefetch(const double* fy, long long ffs, int c, long long e, int n) {
  const FluxSlot s = flux_slot(sizeof(T) == 4, SV, c, ffs);
  if (s.f64) prefetch_l2(fy + s.off + e, n);
  else prefetch_l2(reinterpret_cast<const float*>(fy) + s.off + e, n);
}

constexpr int NF_FACE = 20;   // 5 primitive slots + 14 conserved + the normal current

template <int RM, int SOLVER, int ROWS>
struct FaceGeom {
  static constexpr int R = MPR<RM>::R;
  static constexpr int NS = 2 * R + 2;                 // stencil points
  static constexpr int LONG = 32 + 2 * R + 1;          // staged cells along a 32-face segment
  static constexpr int DEEP = ROWS + 2 * R + 1;        // staged rows across ROWS faces
  // coupled fields: v for the superluminal fall-back (HLL, HLLC), + rho for
  // the HLLC density chain; the HLLE routine couples nothing
  static constexpr int NC = (SOLVER == 7) ? 4 : (SOLVER == 5 ? 3 : 0);
  // D = 0: normal [row][f][LONG], transverse [f][DEEP][32]
  // D = 1: normal [f][DEEP][32],  transverse [row][f][LONG]
  static constexpr int NORMAL0 = ROWS * NF_FACE * LONG;
  static constexpr int NORMAL1 = NF_FACE * DEEP * 32;
  static constexpr int TRANS0 = NC * DEEP * 32;
  static constexpr int TRANS1 = ROWS * NC * LONG;
  static constexpr __host__ __device__ int normal(int D) { return D == 0 ? NORMAL0 : NORMAL1; }
  static constexpr size_t bytes(int D) {
    return sizeof(double) * (size_t)(D == 0 ? NORMAL0 + TRANS0 : NORMAL1 + TRANS1);
  }
  // staged offset of field f at the face's stencil point q (normal) and of
  // coupled field f at stencil point q through the face's cell (transverse)
  template <int D> static __device__ __forceinline__ int nrm(int f, int q, int w, int lane) {
    return D == 0 ? (w * NF_FACE + f) * LONG + lane + q : (f * DEEP + w + q) * 32 + lane;
  }
  template <int D> static __device__ __forceinline__ int trn(int f, int q, int w, int lane) {
    return D == 0 ? (f * DEEP + w + q) * 32 + lane : (w * NC + f) * LONG + lane + q;
  }
};

// staged field f: 0-4 primitive slots (vx, vy, vz, p, rho) of time n, 5-18
// the stage's conserved psi..Sz, 19 the current along the normal
template <int D>
__device__ __forceinline__ const double* face_field(const double* prim, const double* Q, long long fs, int f) {
  if (f < 5) {
    const int pf = (f < 3) ? P_VX + f : (f == 3 ? P_P : P_RHO);
    return prim + (long long)pf * fs;
  }
  const int qf = (f < 19) ? f - 5 : (D == 0 ? Q_JX : Q_JY);
  return Q + (long long)qf * fs;
}

// issue the cp.async copies of one tile (first face i0, j0; last ilast, jlast);
// cells reaching beyond the last face are not copied
template <int RM, int SOLVER, int D, int ROWS>
__device__ __forceinline__ void stage_tile(const InstDesc& I, const StageArgs& sa, double* sn, double* st, int i0,
                                           int j0, int ilast, int jlast, int tid) {
  using G = FaceGeom<RM, SOLVER, ROWS>;
  constexpr int R = G::R, LONG = G::LONG, DEEP = G::DEEP, NC = G::NC;
  const int imax = I.imax, jmax = I.jmax, pitch = I.pitch, bcx = I.bc_x, bcy = I.bc_y;
  const long long fs = I.fstride;
  const double* __restrict__ prim = I.prim[sa.cur];
  const double* __restrict__ Q = I.stage[sa.qin];
  auto cfield = [&](int c) -> const double* { return prim + (long long)(c < 3 ? P_VX + c : P_RHO) * fs; };
  const int ncell = ilast + R + 1 - (i0 - R) + 1;   // x cells i0-R .. ilast+R+1
  const int nrow = jlast + R + 1 - (j0 - R) + 1;    // y rows j0-R .. jlast+R+1
  // rows j0..jlast, cells along x: the normal stencils (D = 0) or the coupled ones (D = 1)
  for (int e = tid; e < ROWS * LONG; e += 32 * ROWS) {
    const int r = e / LONG, c = e - r * LONG;
    if (j0 + r > jlast || c >= ncell) continue;
    const long long off = (long long)map_idx(j0 + r, jmax, bcy) * pitch + map_idx(i0 - R + c, imax, bcx);
    if constexpr (D == 0) {
#pragma unroll
      for (int f = 0; f < NF_FACE; ++f) cp_async8(sn + (r * NF_FACE + f) * LONG + c, face_field<D>(prim, Q, fs, f) + off);
    } else {
#pragma unroll
      for (int f = 0; f < NC; ++f) cp_async8(st + (r * NC + f) * LONG + c, cfield(f) + off);
    }
  }
  // columns i0..ilast, rows along y: the coupled stencils (D = 0) or the normal ones (D = 1)
  for (int e = tid; e < DEEP * 32; e += 32 * ROWS) {
    const int r = e >> 5, c = e & 31;
    if (r >= nrow || i0 + c > ilast) continue;
    const long long off = (long long)map_idx(j0 - R + r, jmax, bcy) * pitch + map_idx(i0 + c, imax, bcx);
    if constexpr (D == 0) {
#pragma unroll
      for (int f = 0; f < NC; ++f) cp_async8(st + (f * DEEP + r) * 32 + c, cfield(f) + off);
    } else {
#pragma unroll
      for (int f = 0; f < NF_FACE; ++f) cp_async8(sn + (f * DEEP + r) * 32 + c, face_field<D>(prim, Q, fs, f) + off);
    }
  }
}

// HLLC star correction of the psi and phi fluxes (16_hllc_flow_mpx.f95:
// 3485-3520, 3908-4300; 16_hllc_flow_mcl.f95:3530-3620) in FP64 for the
// mixed HLLC routines: F holds the FP64 fixed-speed fluxes of roles 0..7 from
// the FP64 field face values Ld / Rd, V the FP32 contact speed after the
// routine's zero threshold, A the routine's FP32 fluxes (NaN when it failed)
template <int D, typename T>
__device__ __forceinline__ void psiphi_star_f64(const Side<double>& Ld, const Side<double>& Rd, T vstar,
                                                const T* A, double* F) {
  using X = Dir<D>;
  const double h = 0.5, V = double(vstar);
  if (isnan(V)) {
    F[R_PSI] = double(A[R_PSI]);
    F[R_PHI] = double(A[R_PHI]);
    return;
  }
  if (V == 0.0) return;
  const double psi_hll = h * (((Rd.psi + Ld.psi) + X::En(Ld)) - X::En(Rd));
  const double phi_hll = h * (((Rd.phi + Ld.phi) + X::Bn(Ld)) - X::Bn(Rd));
  const double En_f = F[R_EN], Bn_f = F[R_BN];
  const double omV = 1.0 - V, opV = V + 1.0, k = V > 0.0 ? omV : opV;
  const double psiR = (psi_hll - V * En_f) / omV, psiL = (psi_hll + V * En_f) / opV;
  const double phiR = (phi_hll - V * Bn_f) / omV, phiL = (phi_hll + V * Bn_f) / opV;
  F[R_PSI] = F[R_PSI] + (k * (psiR - psiL)) * h;
  F[R_PHI] = F[R_PHI] + (k * (phiR - phiL)) * h;
}

// Stencil values of a face of the split tiles: staged field f at normal
// stencil point q (n), coupled field f at point q through the face's cell (t)
template <int RM, int SOLVER, int D, int ROWS>
struct SplitAcc {
  using G = FaceGeom<RM, SOLVER, ROWS>;
  const double* sn;
  const double* st;
  int w, lane;
  __device__ __forceinline__ double n(int f, int q) const { return sn[G::template nrm<D>(f, q, w, lane)]; }
  __device__ __forceinline__ double t(int f, int q) const { return st[G::template trn<D>(f, q, w, lane)]; }
};

// Face values of the primitive slots v, p, rho of one face, with the
// superluminal fall-back and the density fix-ups already applied (the fused
// stage kernel forms them once for the x and the y face of a point)
template <typename T>
struct FacePre {
  T vL[3], vR[3], pL, pR, rhoL, rhoR;
  T dpL, dpR;    // split-pressure solvers: pL, pR minus pc0
  double pc0;    // the face's FP64 reference pressure (cell i / j of the face)
};

// Mixed-precision HLL / HLLE / HLLC of the MP routines split the pressure:
// p is reconstructed as differences from the FP64 pressure pc0 of the face's
// cell (the MP limiter and its positivity fix are translation-equivariant),
// the FP32 normal momentum flux carries p - pc0, and pc0 is added back to
// that flux in FP64.  The pressure (~1 in the KH layer) would otherwise be
// rounded to FP32 in the flux whose divergence drives the small normal
// velocity of the perturbation.
template <typename T, int SV>
constexpr bool kSplitP = kEmF64<T, SV> && mixed_split_p(SV);

// flux of one face from its stencil accessor (16_hll_flow_mpx.f95 /
// 16_hllc_flow_mpx.f95 for one interface); returns status bits.  With PRE
// the primitive slots come from *pre instead of being reconstructed here.
template <int RM, int SOLVER, typename T, int D, bool PRE, class ACC>
__device__ __forceinline__ uint32_t face_flux(const ACC& acc, const FacePre<T>* pre, double gamma_d, double sigma_d,
                                              flux_t<T, SOLVER> (&F)[NROLE]) {
  constexpr int R = MPR<RM>::R, NS = 2 * R + 2;
  auto nrmd = [&](int f, int q) -> double { return acc.n(f, q); };
  auto nrm = [&](int f, int q) -> T { return T(nrmd(f, q)); };
  auto trn = [&](int f, int q) -> T { return T(acc.t(f, q)); };
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
  Side<double> Ld{}, Rd{};   // FP64 field face values (mixed routines with FP64 field fluxes)
  double pc0 = 0.0;          // reference pressure of the split-pressure solvers
  if constexpr (SOLVER == 1) {
    // Lax-Friedrichs with MC slopes, 15_lax_flow.f95:920-1457: for stencil
    // cells 0..3 (the face lies between 1 and 2)
    //   L = p1 + FAC mcl(p2 - p1, p1 - p0),  R = m2 - FAC mcl(p3 - p2, p2 - p1),
    // both with the slopes of p, and the face flux 0.5 (L + R), negated for
    // the sign-flipped roles R_BT1 and R_ET2
    static_assert(RM == 3, "the Lax fluxes use the MC slopes");
    const T gamma = T(gamma_d);
    auto cell = [&](int q) {
      Side<T> s;
      s.vx = nrm(0, q); s.vy = nrm(1, q); s.vz = nrm(2, q); s.p = nrm(3, q); s.rho = nrm(4, q);
      s.psi = nrm(5 + Q_PSI, q); s.phi = nrm(5 + Q_PHI, q);
      s.Ex = nrm(5 + Q_EX, q); s.Ey = nrm(5 + Q_EY, q); s.Ez = nrm(5 + Q_EZ, q);
      s.Bx = nrm(5 + Q_BX, q); s.By = nrm(5 + Q_BY, q); s.Bz = nrm(5 + Q_BZ, q);
      s.q = nrm(5 + Q_Q, q); s.D = nrm(5 + Q_D, q); s.tau = nrm(5 + Q_TAU, q);
      s.Sx = nrm(5 + Q_SX, q); s.Sy = nrm(5 + Q_SY, q); s.Sz = nrm(5 + Q_SZ, q);
      s.J = nrm(19, q);
      return s;
    };
    T hW2[NS], EB[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) lax_cell_scalars(cell(q), gamma, hW2[q], EB[q]);
    if constexpr (kEmF64<T, SOLVER>) {
      // mixed precision: the field roles (psi, phi, E, B) form p = F + U in
      // FP64, take the MC slopes of the differences from p of cell 1 in FP32
      // (the slopes are differences) and the face flux back in FP64
      auto cell_d = [&](int q) {
        Side<double> sd{};
        sd.psi = nrmd(5 + Q_PSI, q); sd.phi = nrmd(5 + Q_PHI, q);
        sd.Ex = nrmd(5 + Q_EX, q); sd.Ey = nrmd(5 + Q_EY, q); sd.Ez = nrmd(5 + Q_EZ, q);
        sd.Bx = nrmd(5 + Q_BX, q); sd.By = nrmd(5 + Q_BY, q); sd.Bz = nrmd(5 + Q_BZ, q);
        return sd;
      };
#pragma unroll
      for (int r = R_PSI; r <= R_ET2; ++r) {
        double pd[NS], m2 = 0.0;
#pragma unroll
        for (int q = 0; q < NS; ++q) {
          double f, u;
          lax_pair<D>(r, cell_d(q), 0.0, 0.0, f, u);
          pd[q] = f + u;
          if (q == 2) m2 = f - u;
        }
        const double c0 = pd[1];
        T d[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) d[q] = T(pd[q] - c0);
        const double Lf = c0 + double(d[1] + T(0.5) * mc_slope(d[2] - d[1], d[1] - d[0]));
        const double Rf = m2 - double(T(0.5) * mc_slope(d[3] - d[2], d[2] - d[1]));
        F[r] = (r == R_BT1 || r == R_ET2) ? -(0.5 * (Lf + Rf)) : 0.5 * (Lf + Rf);
      }
    }
#pragma unroll
    for (int r = (kEmF64<T, SOLVER> ? R_Q : 0); r < NROLE; ++r) {
      T p[NS], m2 = T(0);
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        T f, u;
        lax_pair<D>(r, cell(q), hW2[q], EB[q], f, u);
        p[q] = f + u;
        if (q == 2) m2 = f - u;
      }
      const T Lf = p[1] + T(0.5) * mc_slope(p[2] - p[1], p[1] - p[0]);
      const T Rf = m2 - T(0.5) * mc_slope(p[3] - p[2], p[2] - p[1]);
      F[r] = (r == R_BT1 || r == R_ET2) ? -(T(0.5) * (Lf + Rf)) : T(0.5) * (Lf + Rf);
    }
    return stt;
  }
  if constexpr (SOLVER >= 2 && SOLVER <= 4) {
    // HLL (16_hll_flow_mcl.f95:565-1396), HLLE (16_hlle_flow_mcl.f95:1647-4345)
    // or HLLC (16_hllc_flow_mcl.f95:1760-4056) with the second-order MC
    // reconstruction (x and y faces of a point are the same formulas in the
    // direction roles)
    static_assert(RM == 3, "the MCL fluxes use the MC reconstruction");
    T m_et2[2], m_bt1[2];   // "_m" values (-u + slope) of E_t2 and B_t1, left and right
    auto recm = [&](int f, T& Lv, T& Rv, T* m) {
      T u[NS];
#pragma unroll
      for (int q = 0; q < NS; ++q) u[q] = nrm(f, q);
      const T sl = T(0.5) * mc_slope(u[2] - u[1], u[1] - u[0]);
      const T sr = T(0.5) * mc_slope(u[3] - u[2], u[2] - u[1]);
      Lv = u[1] + sl;
      Rv = u[2] - sr;
      if (m) { m[0] = -u[1] + sl; m[1] = -u[2] - sr; }
    };
    constexpr int fEt2 = 5 + (D == 0 ? Q_EZ : Q_EX), fBt1 = 5 + (D == 0 ? Q_BY : Q_BZ);
    recm(0, L.vx, Rs.vx, nullptr);
    recm(1, L.vy, Rs.vy, nullptr);
    recm(2, L.vz, Rs.vz, nullptr);
    recm(3, L.p, Rs.p, nullptr);
    recm(4, L.rho, Rs.rho, nullptr);
    if constexpr (kEmF64<T, SOLVER>) {
      // mixed precision: the field slots as differences from the FP64 value
      // of stencil cell 1 (the MC slopes are differences), face and "_m"
      // values back in FP64, their fluxes in FP64 (see the MP routines)
      double md_et2[2], md_bt1[2];
      auto recm_delta = [&](int f, double& Lv, double& Rv, double* m) {
        const double c0 = nrmd(f, 1);
        T u[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) u[q] = T(nrmd(f, q) - c0);
        const T sl = T(0.5) * mc_slope(u[2] - u[1], u[1] - u[0]);
        const T sr = T(0.5) * mc_slope(u[3] - u[2], u[2] - u[1]);
        Lv = c0 + double(u[1] + sl);
        Rv = c0 + double(u[2] - sr);
        if (m) { m[0] = -(c0 + double(u[1])) + double(sl); m[1] = -(c0 + double(u[2])) - double(sr); }
      };
      recm_delta(5 + Q_PSI, Ld.psi, Rd.psi, nullptr);
      recm_delta(5 + Q_PHI, Ld.phi, Rd.phi, nullptr);
      recm_delta(5 + Q_EX, Ld.Ex, Rd.Ex, fEt2 == 5 + Q_EX ? md_et2 : nullptr);
      recm_delta(5 + Q_EY, Ld.Ey, Rd.Ey, nullptr);
      recm_delta(5 + Q_EZ, Ld.Ez, Rd.Ez, fEt2 == 5 + Q_EZ ? md_et2 : nullptr);
      recm_delta(5 + Q_BX, Ld.Bx, Rd.Bx, nullptr);
      recm_delta(5 + Q_BY, Ld.By, Rd.By, fBt1 == 5 + Q_BY ? md_bt1 : nullptr);
      recm_delta(5 + Q_BZ, Ld.Bz, Rd.Bz, fBt1 == 5 + Q_BZ ? md_bt1 : nullptr);
      double Ad[NROLE];
      mcl_fluxes<D>(Ld, Rd, md_et2, md_bt1, gamma_d, sigma_d, Ad);   // roles 0..7 used
#pragma unroll
      for (int c = R_PSI; c <= R_ET2; ++c) F[c] = Ad[c];
      L.psi = T(Ld.psi); L.phi = T(Ld.phi); L.Ex = T(Ld.Ex); L.Ey = T(Ld.Ey); L.Ez = T(Ld.Ez);
      L.Bx = T(Ld.Bx); L.By = T(Ld.By); L.Bz = T(Ld.Bz);
      Rs.psi = T(Rd.psi); Rs.phi = T(Rd.phi); Rs.Ex = T(Rd.Ex); Rs.Ey = T(Rd.Ey); Rs.Ez = T(Rd.Ez);
      Rs.Bx = T(Rd.Bx); Rs.By = T(Rd.By); Rs.Bz = T(Rd.Bz);
      m_et2[0] = T(md_et2[0]); m_et2[1] = T(md_et2[1]);
      m_bt1[0] = T(md_bt1[0]); m_bt1[1] = T(md_bt1[1]);
    } else {
      recm(5 + Q_PSI, L.psi, Rs.psi, nullptr);
      recm(5 + Q_PHI, L.phi, Rs.phi, nullptr);
      recm(5 + Q_EX, L.Ex, Rs.Ex, fEt2 == 5 + Q_EX ? m_et2 : nullptr);
      recm(5 + Q_EY, L.Ey, Rs.Ey, nullptr);
      recm(5 + Q_EZ, L.Ez, Rs.Ez, fEt2 == 5 + Q_EZ ? m_et2 : nullptr);
      recm(5 + Q_BX, L.Bx, Rs.Bx, nullptr);
      recm(5 + Q_BY, L.By, Rs.By, fBt1 == 5 + Q_BY ? m_bt1 : nullptr);
      recm(5 + Q_BZ, L.Bz, Rs.Bz, fBt1 == 5 + Q_BZ ? m_bt1 : nullptr);
    }
    recm(5 + Q_Q, L.q, Rs.q, nullptr);
    recm(5 + Q_D, L.D, Rs.D, nullptr);
    recm(5 + Q_TAU, L.tau, Rs.tau, nullptr);
    recm(5 + Q_SX, L.Sx, Rs.Sx, nullptr);
    recm(5 + Q_SY, L.Sy, Rs.Sy, nullptr);
    recm(5 + Q_SZ, L.Sz, Rs.Sz, nullptr);
    T vstar = T(0);
    auto riemann_mc = [&](T* A) {
      if constexpr (SOLVER == 2) mcl_fluxes<D>(L, Rs, m_et2, m_bt1, T(gamma_d), T(sigma_d), A);
      else if constexpr (SOLVER == 3) hllemc_fluxes<D>(L, Rs, m_et2, m_bt1, T(gamma_d), T(sigma_d), A, stt);
      else hllcmc_fluxes<D>(L, Rs, m_et2, m_bt1, T(gamma_d), T(sigma_d), A, stt,
                            kEmF64<T, SOLVER> ? &vstar : nullptr);
    };
    if constexpr (kEmF64<T, SOLVER>) {
      T A[NROLE];
      riemann_mc(A);
#pragma unroll
      for (int c = R_Q; c < NROLE; ++c) F[c] = double(A[c]);
      if constexpr (SOLVER == 4) psiphi_star_f64<D>(Ld, Rd, vstar, A, F);
    } else {
      riemann_mc(F);
    }
    return stt;
  }
  // primitive slots of this direction (21-25 for x, 58-62 for y)
  if constexpr (PRE) {
    L.vx = pre->vL[0]; L.vy = pre->vL[1]; L.vz = pre->vL[2];
    Rs.vx = pre->vR[0]; Rs.vy = pre->vR[1]; Rs.vz = pre->vR[2];
    L.p = pre->pL; Rs.p = pre->pR;
    L.rho = pre->rhoL; Rs.rho = pre->rhoR;
    if constexpr (kSplitP<T, SOLVER>) { L.dp = pre->dpL; Rs.dp = pre->dpR; pc0 = pre->pc0; }
  } else {
    rec(0, L.vx, Rs.vx);
    rec(1, L.vy, Rs.vy);
    rec(2, L.vz, Rs.vz);
    if constexpr (kSplitP<T, SOLVER>) {
      pc0 = nrmd(3, R);
      T u[NS];
#pragma unroll
      for (int q = 0; q < NS; ++q) u[q] = T(nrmd(3, q) - pc0);
      const Pair<T> pp = MPCall<RM, T>::call_posd(u, pc0);
      L.dp = pp.L; Rs.dp = pp.R;
      L.p = T(pc0 + double(pp.L)); Rs.p = T(pc0 + double(pp.R));
    } else {
      recp(3, L.p, Rs.p);
    }
    recp(4, L.rho, Rs.rho);
  }
  if constexpr (!PRE && (SOLVER == 5 || SOLVER == 7)) {
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
  if constexpr (!PRE && SOLVER == 7) {
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
  if constexpr (kEmF64<T, SOLVER>) {
    // mixed precision: psi, phi, E and B are reconstructed as differences
    // from the cell's FP64 value (the MP limiters are translation-equivariant:
    // weights summing to 1, limiter tests on differences), so the FP32
    // rounding is relative to the local variation rather than to the
    // background field; their fluxes, linear in these face values (plus the
    // HLLC star correction of psi and phi, below), are formed in FP64
    auto rec_delta = [&](int f, double& Lv, double& Rv) {
      const double c0 = nrmd(f, R);
      T u[NS];
#pragma unroll
      for (int q = 0; q < NS; ++q) u[q] = T(nrmd(f, q) - c0);
      const Pair<T> p = MPCall<RM, T>::template call<false>(u);
      Lv = c0 + double(p.L); Rv = c0 + double(p.R);
    };
    rec_delta(5 + Q_PSI, Ld.psi, Rd.psi);
    rec_delta(5 + Q_PHI, Ld.phi, Rd.phi);
    rec_delta(5 + Q_EX, Ld.Ex, Rd.Ex);
    rec_delta(5 + Q_EY, Ld.Ey, Rd.Ey);
    rec_delta(5 + Q_EZ, Ld.Ez, Rd.Ez);
    rec_delta(5 + Q_BX, Ld.Bx, Rd.Bx);
    rec_delta(5 + Q_BY, Ld.By, Rd.By);
    rec_delta(5 + Q_BZ, Ld.Bz, Rd.Bz);
    double Ad[NROLE];
    em_fluxes<D>(Ld, Rd, Ad);
#pragma unroll
    for (int c = R_PSI; c <= R_ET2; ++c) F[c] = Ad[c];
    L.psi = T(Ld.psi); L.phi = T(Ld.phi); L.Ex = T(Ld.Ex); L.Ey = T(Ld.Ey); L.Ez = T(Ld.Ez);
    L.Bx = T(Ld.Bx); L.By = T(Ld.By); L.Bz = T(Ld.Bz);
    Rs.psi = T(Rd.psi); Rs.phi = T(Rd.phi); Rs.Ex = T(Rd.Ex); Rs.Ey = T(Rd.Ey); Rs.Ez = T(Rd.Ez);
    Rs.Bx = T(Rd.Bx); Rs.By = T(Rd.By); Rs.Bz = T(Rd.Bz);
  } else {
    rec(5 + Q_PSI, L.psi, Rs.psi);
    rec(5 + Q_PHI, L.phi, Rs.phi);
    rec(5 + Q_EX, L.Ex, Rs.Ex);
    rec(5 + Q_EY, L.Ey, Rs.Ey);
    rec(5 + Q_EZ, L.Ez, Rs.Ez);
    rec(5 + Q_BX, L.Bx, Rs.Bx);
    rec(5 + Q_BY, L.By, Rs.By);
    rec(5 + Q_BZ, L.Bz, Rs.Bz);
  }
  rec(5 + Q_Q, L.q, Rs.q);
  rec(5 + Q_D, L.D, Rs.D);
  rec(5 + Q_TAU, L.tau, Rs.tau);
  rec(5 + Q_SX, L.Sx, Rs.Sx);
  rec(5 + Q_SY, L.Sy, Rs.Sy);
  rec(5 + Q_SZ, L.Sz, Rs.Sz);
  rec(19, L.J, Rs.J);
  const T gamma = T(gamma_d);
  T vstar = T(0);
  constexpr bool PS = kSplitP<T, SOLVER>;
  auto riemann = [&](T* A) {
    if constexpr (SOLVER == 5) hll_fluxes<D, PS>(L, Rs, gamma, A);
    else if constexpr (SOLVER == 6) hlle_fluxes<D, PS>(L, Rs, gamma, A, stt, T(pc0));
    else if constexpr (SOLVER == 7)
      hllc_fluxes<D, PS>(L, Rs, gamma, A, stt, kEmF64<T, SOLVER> ? &vstar : nullptr, T(pc0));
  };
  if constexpr (kEmF64<T, SOLVER>) {
    T A[NROLE];
    riemann(A);
#pragma unroll
    for (int c = R_Q; c < NROLE; ++c) F[c] = double(A[c]);
    if constexpr (PS) F[R_SN] = pc0 + double(A[R_SN]);
    if constexpr (SOLVER == 7) psiphi_star_f64<D>(Ld, Rd, vstar, A, F);
  } else {
    riemann(F);
  }
  return stt;
}

__device__ __forceinline__ const InstDesc& tile_inst(const InstDesc* __restrict__ insts, int ninst, int kind, int& b) {
  int k = 0;
  for (int t = 1; t < ninst; ++t)
    if (insts[t].block_begin[kind] <= b) k = t;
  b -= insts[k].block_begin[kind];
  return insts[k];
}

// Tile loop: CTA b handles tiles b, b + gridDim.x, ... of the launch (ntiles
// over all instances), so a grid of one CTA per tile and a persistent grid
// of a few CTAs per SM run the same code.

// y faces: 32 columns x ROWS face rows j = j0-1+warp in [-1, jmax]; writes
// Fy(i, j+1/2) to the flux scratch
template <int RM, int SOLVER, typename T, int ROWS>
__global__ void __launch_bounds__(32 * ROWS, 16 / ROWS)
k_yface(const InstDesc* __restrict__ insts, int ninst, int ntiles, StageArgs sa) {
  using G = FaceGeom<RM, SOLVER, ROWS>;
  extern __shared__ double smem[];
  const int lane = threadIdx.x, w = threadIdx.y;
  double* sn = smem;
  double* st = smem + G::normal(1);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int b = tile;
    const InstDesc& I = tile_inst(insts, ninst, LK_YFACE, b);
    const int bpr = (I.imax + 1 + 31) / 32;
    const int i0 = (b % bpr) * 32, j0 = (b / bpr) * ROWS - 1;
    const int ilast = min(i0 + 31, I.imax), jlast = min(j0 + ROWS - 1, I.jmax);
    stage_tile<RM, SOLVER, 1, ROWS>(I, sa, sn, st, i0, j0, ilast, jlast, w * 32 + lane);
    cp_async_wait_all();
    __syncthreads();
    const int i = i0 + lane, j = j0 + w;
    if (i <= ilast && j <= jlast) {
      flux_t<T, SOLVER> F[NROLE];
      const SplitAcc<RM, SOLVER, 1, ROWS> acc{sn, st, w, lane};
      const uint32_t stt = face_flux<RM, SOLVER, T, 1, false>(acc, (const FacePre<T>*)nullptr, I.gamma, I.sigma, F);
      const long long fo = (long long)(j + 1) * I.fpitch + i;
#pragma unroll
      for (int c = 0; c < NROLE; ++c) flux_store<T, SOLVER>(I.fy, I.ffs, c, fo, double(F[c]));
      if (stt) atomicOr(I.status, stt);
    }
    __syncthreads();   // the next tile's copies overwrite the staged values
  }
}

// ------------------------------------------------- x faces + point update
// EP selects the epilogue: EP_RHS stores the stage right-hand side only (the
// routine mirror), EP_MID prepares stage l+1, EP_LAST finishes the step.
enum Epilogue { EP_RHS = 0, EP_MID = 1, EP_LAST = 2 };

// centre values of stage l (psi, phi, E, B, q) and time n (v) of a point
struct Centre { double q, psi, phi, Ex, Ey, Ez, Bx, By, Bz, vx, vy, vz; };

// flux divergence + sources of point (i, j) (17_fluxandsource.f95:441-635)
// and the fused epilogue; qx[r] = (Fx(i+1/2) - Fx(i-1/2)) / delx per role,
// fyd(r) = Fy(j+1/2) - Fy(j-1/2) per role
// valid == false (EP_LAST only): the lane computes a copy of a real point so
// that its warp reaches con2prim converged, and stores nothing
template <int EP, typename T, int SV, class FYD>
__device__ __forceinline__ uint32_t update_point(const InstDesc& I, const StageArgs& sa, int i, int j,
                                                 const double (&qx)[NROLE], const FYD& fyd, const Centre& cv,
                                                 bool valid = true) {
  const int pitch = I.pitch;
  const long long fs = I.fstride;
  const double* __restrict__ prim = I.prim[sa.cur];
  const double* __restrict__ aux = I.aux[sa.cur];
  uint32_t st = 0;
  const long long pc = (long long)j * pitch + i;
  const double dly = I.dely, iy2 = I.inv_dely_pow2;
  auto qy = [&](int r) {   // (dy)/dly
    const double d = fyd(r);
    return iy2 != 0.0 ? d * iy2 : d / dly;
  };
  auto qxf = [&](int r) { return qx[r]; };
  const double q = cv.q, psi = cv.psi, phi = cv.phi, Ex = cv.Ex, Ey = cv.Ey, Ez = cv.Ez;
  const double Bx = cv.Bx, By = cv.By, Bz = cv.Bz, vx = cv.vx, vy = cv.vy, vz = cv.vz;
  const double W = aux[A_W * fs + pc];
  double K[NRHS];
  // 17_fluxandsource.f95:488-598; z differences are (X - X)/Delz = 0
  // (-a)/d == -(a/d) exactly, so every term is -/+ the quotient of a difference
  K[Q_PSI] = -qxf(R_PSI) - qy(R_PSI) + q - I.kappa_psi * psi;
  K[Q_PHI] = -qxf(R_PHI) - qy(R_PHI) - I.kappa_phi * phi;
  K[Q_BX] = -qy(R_BT2) + 0.0 - qxf(R_BN);
  K[Q_BY] = qxf(R_BT1) - qy(R_BN);
  K[Q_BZ] = -qxf(R_BT2) + qy(R_BT1);
  K[Q_EX] = qy(R_ET2) - qxf(R_EN) - q * vx;
  K[Q_EY] = 0.0 - qxf(R_ET1) - qy(R_EN) - q * vy;
  K[Q_EZ] = qxf(R_ET2) - qy(R_ET1) - q * vz;
  K[Q_Q] = -qxf(R_Q) - qy(R_Q);
  K[Q_D] = -qxf(R_D) - qy(R_D);
  K[Q_TAU] = -qxf(R_TAU) - qy(R_TAU);
  K[Q_SX] = -qxf(R_SN) - qy(R_ST2);
  K[Q_SY] = -qxf(R_ST1) - qy(R_SN);
  K[Q_SZ] = -qxf(R_ST2) - qy(R_ST1);
  stiff_source(I.sigma, W, vx, vy, vz, Ex, Ey, Ez, Bx, By, Bz, K[K_SEX], K[K_SEY], K[K_SEZ]);

  if constexpr (EP == EP_RHS) {
#pragma unroll
    for (int c = 0; c < NRHS; ++c) I.rhs_out[c * fs + pc] = K[c];
  } else {
    // sumfin, 18_sumfin.f95:20-66
    double fin[NCONS];
#pragma unroll
    for (int c = 0; c < NCONS; ++c) {
      // sums of stages with zero weights are zero (up to the sign of zero)
      const double prev = sa.fin_load ? I.finsum[c * fs + pc] : 0.0;
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
      if (sa.fin_store) {
#pragma unroll
        for (int c = 0; c < NCONS; ++c) I.finsum[c * fs + pc] = fin[c];
      }
      // sumint for stage l+1 (09_sumint.f95:18-67); intsum is zeroed only
      // once per step (07_clean_var.f95), so it accumulates across stages
      double acc[NCONS];
#pragma unroll
      for (int c = 0; c < NCONS; ++c) acc[c] = sa.need_intsum_load ? I.intsum[c * fs + pc] : 0.0;
      for (int m = 1; m <= sa.l; ++m) {
        const double ab = sa.ab_next[m - 1], abt = sa.abt_next[m - 1];
        if (ab == 0.0 && abt == 0.0) continue;
        const double* Km = (m < sa.l) ? I.kbuf + (long long)sa.kslot[m - 1] * NRHS * fs : nullptr;
        // with Ab = 0 the term ab * F is a zero: the flux of K_m is not read
        // (a stored K_m may hold its E sources only), which changes at most
        // the sign of a zero sum
#pragma unroll
        for (int c = 0; c < NCONS; ++c) {
          if (c >= Q_EX && c <= Q_EZ) {
            const double S = Km ? Km[(K_SEX + c - Q_EX) * fs + pc] : K[K_SEX + c - Q_EX];
            if (ab == 0.0) {
              acc[c] = acc[c] + (0.0 - abt * S);
            } else {
              const double F = Km ? Km[c * fs + pc] : K[c];
              acc[c] = acc[c] + (ab * F - abt * S);
            }
          } else if (ab != 0.0) {
            const double F = Km ? Km[c * fs + pc] : K[c];
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
        for (int c = 0; c < NRHS; ++c)
          if (!sa.store_k_src || c >= K_SEX) Ko[c * fs + pc] = K[c];
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
      // varfin's D and tau, which the run diagnostics read (con2prim does not write them back)
      if (sa.diag_cons != nullptr && valid) { sa.diag_cons[pc] = Un[Q_D]; sa.diag_cons[fs + pc] = Un[Q_TAU]; }
      if (I.c2p == 2 && I.c2p_tc) {
        // con2prim follows in k_c2p_step: the evolved D, tau, S go to the
        // final-sum slabs (read above, not needed again this step), the
        // fields varfin completes to the primitives of time n+1
        if (!valid) return 0u;
#pragma unroll
        for (int c = Q_D; c <= Q_SZ; ++c) I.finsum[c * fs + pc] = Un[c];
        double* po = I.prim[1 - sa.cur];
        po[P_PSI * fs + pc] = Un[Q_PSI]; po[P_PHI * fs + pc] = Un[Q_PHI];
        po[P_EX * fs + pc] = Un[Q_EX]; po[P_EY * fs + pc] = Un[Q_EY]; po[P_EZ * fs + pc] = Un[Q_EZ];
        po[P_BX * fs + pc] = Un[Q_BX]; po[P_BY * fs + pc] = Un[Q_BY]; po[P_BZ * fs + pc] = Un[Q_BZ];
        po[P_Q * fs + pc] = Un[Q_Q];
        return st;
      }
      // con2prim, l_swap = 1 (main_cueva_code.f95:312-326)
      C2PIn in{Un[Q_D], Un[Q_TAU], Un[Q_SX], Un[Q_SY], Un[Q_SZ], Un[Q_EX], Un[Q_EY], Un[Q_EZ],
               Un[Q_BX], Un[Q_BY], Un[Q_BZ], vx, vy, vz, prim[P_RHO * fs + pc], prim[P_P * fs + pc]};
      C2POut o;
      st |= c2p_dispatch(I, in, o, valid, I.c2p == 2);   // k_xupd sends whole warps for c2p = 2
      if (!valid) return 0u;
      double pv[NPRIM];
      pv[P_RHO] = o.rho; pv[P_P] = o.p; pv[P_VX] = o.vx; pv[P_VY] = o.vy; pv[P_VZ] = o.vz;
      pv[P_PSI] = Un[Q_PSI]; pv[P_PHI] = Un[Q_PHI];
      pv[P_EX] = Un[Q_EX]; pv[P_EY] = Un[Q_EY]; pv[P_EZ] = Un[Q_EZ];
      pv[P_BX] = Un[Q_BX]; pv[P_BY] = Un[Q_BY]; pv[P_BZ] = Un[Q_BZ]; pv[P_Q] = Un[Q_Q];
      double* po = I.prim[1 - sa.cur];
#pragma unroll
      for (int c = 0; c < NPRIM; ++c) po[c * fs + pc] = pv[c];
      // with the primitive reconstruction the next step starts in k_recons_begin
      if (!I.primitive_rec) begin_step_point(I, sa.abt_diag_first, I.aux[1 - sa.cur], I.stage[1 - sa.qin], pc, pv);
    }
  }
  return st;
}

// L2 prefetch of the update's other inputs for the points i0+1 .. ilast of
// rows j0 .. jl: the 6 aux and 9 time-n primitive fields, the final sums and
// stage sums when loaded, and the stored stage right-hand sides a later row
// reads (their E sources only where that row's Ab is zero)
__device__ __forceinline__ void prefetch_update_rows(const InstDesc& I, const StageArgs& sa, int i0, int ilast, int j0,
                                                     int jl, int tid, int nthr) {
  const long long fs = I.fstride;
  const int npt = ilast - i0, nr = jl - j0 + 1;
  if (npt <= 0 || nr <= 0) return;
  const int nfin = sa.fin_load ? NCONS : 0, nint = sa.need_intsum_load ? NCONS : 0;
  int nkf = 0;   // stored K fields read
  for (int m = 1; m < sa.l; ++m)
    if (sa.kslot[m - 1] >= 0) nkf += sa.ab_next[m - 1] != 0.0 ? NRHS : (sa.abt_next[m - 1] != 0.0 ? 3 : 0);
  const int ncen = NAUX + 9 + nfin + nint + nkf;
  for (int e = tid; e < ncen * nr; e += nthr) {
    const int r = e % nr;
    int f = e / nr;
    const double* base;
    if (f < NAUX) base = I.aux[sa.cur] + f * fs;
    else if ((f -= NAUX) < 9) base = I.prim[sa.cur] + (P_PSI + f) * fs;
    else if ((f -= 9) < nfin) base = I.finsum + f * fs;
    else if ((f -= nfin) < nint) base = I.intsum + f * fs;
    else {
      f -= nint;
      base = nullptr;
      for (int m = 1; m < sa.l && !base; ++m) {
        if (sa.kslot[m - 1] < 0) continue;
        const int nm = sa.ab_next[m - 1] != 0.0 ? NRHS : (sa.abt_next[m - 1] != 0.0 ? 3 : 0);
        if (f < nm) base = I.kbuf + ((long long)sa.kslot[m - 1] * NRHS + (nm == NRHS ? f : K_SEX + f)) * fs;
        else f -= nm;
      }
      if (!base) continue;
    }
    prefetch_l2(base + (long long)(j0 + r) * I.pitch + i0 + 1, npt);
  }
}

template <int RM, int SOLVER, typename T, int EP, int ROWS>
__device__ __forceinline__ void xupd_tile(const InstDesc& I, const StageArgs& sa, int b, double* sn, double* st) {
  using G = FaceGeom<RM, SOLVER, ROWS>;
  constexpr int R = G::R, LONG = G::LONG;
  const int lane = threadIdx.x, w = threadIdx.y;
  // a tile updates 31 points per row: faces i0 .. i0+31 (i0 = first point - 1)
  const int bpr = (I.imax + 1 + 30) / 31;
  const int i0 = (b % bpr) * 31 - 1, j0 = (b / bpr) * ROWS;
  const int ilast = min(i0 + 31, I.imax), jlast = min(j0 + ROWS - 1, I.jmax);
  stage_tile<RM, SOLVER, 0, ROWS>(I, sa, sn, st, i0, j0, ilast, jlast, w * 32 + lane);
  if constexpr (EP != EP_RHS) {
    // the update's other inputs and the y fluxes go to L2 while the faces
    // are computed
    prefetch_update_rows(I, sa, i0, ilast, j0, jlast, w * 32 + lane, 32 * ROWS);
    const int npt = ilast - i0, nr = jlast - j0 + 1;
    for (int e = w * 32 + lane; e < NROLE * (nr + 1) && npt > 0; e += 32 * ROWS) {
      const int r = e % (nr + 1), c = e / (nr + 1);
      flux_prefetch<T, SOLVER>(I.fy, I.ffs, c, (long long)(j0 + r) * I.fpitch + i0 + 1, npt);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  const int i = i0 + lane, j = j0 + w;
  if (j > jlast) return;   // whole warp; the caller synchronises before the next tile
  flux_t<T, SOLVER> F[NROLE];
#pragma unroll
  for (int c = 0; c < NROLE; ++c) F[c] = 0;
  uint32_t stt = 0;
  if (i <= ilast) {
    const SplitAcc<RM, SOLVER, 0, ROWS> acc{sn, st, w, lane};
    stt = face_flux<RM, SOLVER, T, 0, false>(acc, (const FacePre<T>*)nullptr, I.gamma, I.sigma, F);
  }
  if constexpr (EP == EP_RHS) {
    // the routine mirror of the flux routine (mode 2) also stores the x-face
    // fluxes; a face on a tile seam is stored by the tile of its right point
    if (sa.mode == 2 && i <= ilast && (lane >= 1 || i == -1)) {
#pragma unroll
      for (int c = 0; c < NROLE; ++c) I.fx[c * I.ffs + (long long)j * I.fpitch + (i + 1)] = double(F[c]);
    }
  }
  // Fx(i-1/2) of point i is the face of lane-1
  const double dlx = I.delx, ix2 = I.inv_delx_pow2;
  double qx[NROLE];
#pragma unroll
  for (int c = 0; c < NROLE; ++c) {
    const double fr = double(F[c]);
    const double fl = __shfl_up_sync(0xffffffffu, fr, 1);
    const double d = fr - fl;
    qx[c] = ix2 != 0.0 ? d * ix2 : d / dlx;
  }
  const bool valid = lane >= 1 && i <= ilast;
  // after the last stage every lane of the warp enters the update (lanes
  // without a point repeat a real one and store nothing), so con2prim runs
  // converged; earlier stages update the real points only
  const bool warp_c2p = EP == EP_LAST && I.c2p == 2 && !I.c2p_tc;
  if (valid || warp_c2p) {
    const int ii = valid ? i : (lane == 0 ? i0 + 1 : ilast);
    const int ln = ii - i0;   // staged cell ii is stencil point R of lane ln's face
    if (warp_c2p) {
      // a lane without a point takes the divergence of the point it repeats
#pragma unroll
      for (int c = 0; c < NROLE; ++c) qx[c] = __shfl_sync(0xffffffffu, qx[c], ln);
    }
    auto cs = [&](int f) { return sn[(w * NF_FACE + f) * LONG + ln + R]; };
    const Centre cv{cs(5 + Q_Q), cs(5 + Q_PSI), cs(5 + Q_PHI), cs(5 + Q_EX), cs(5 + Q_EY), cs(5 + Q_EZ),
                    cs(5 + Q_BX), cs(5 + Q_BY), cs(5 + Q_BZ), cs(0), cs(1), cs(2)};
    const long long fyo = (long long)(j + 1) * I.fpitch + ii;   // Fy(ii, j+1/2); Fy(ii, j-1/2) at -fpitch
    auto fyd = [&](int r) {
      return flux_load<T, SOLVER>(I.fy, I.ffs, r, fyo) - flux_load<T, SOLVER>(I.fy, I.ffs, r, fyo - I.fpitch);
    };
    stt |= update_point<EP, T, SOLVER>(I, sa, ii, j, qx, fyd, cv, valid);
  }
  if (stt) atomicOr(I.status, stt);
}

template <int RM, int SOLVER, typename T, int EP, int ROWS>
__global__ void __launch_bounds__(32 * ROWS, 16 / ROWS)
k_xupd(const InstDesc* __restrict__ insts, int ninst, int ntiles, StageArgs sa) {
  using G = FaceGeom<RM, SOLVER, ROWS>;
  extern __shared__ double smem[];
  double* sn = smem;
  double* st = smem + G::normal(0);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int b = tile;
    const InstDesc& I = tile_inst(insts, ninst, LK_XUPD, b);
    xupd_tile<RM, SOLVER, T, EP, ROWS>(I, sa, b, sn, st);
    __syncthreads();   // the next tile's copies overwrite the staged values
  }
}

// ------------------------------------------------------- fused stage kernel
// k_stage: one launch per RK stage.  A CTA of 32 x ROWS threads owns a strip
// of 31 points along x (lane 0 carries the strip's left face) and marches up
// a segment of I.seg_rows grid rows in bands of ROWS rows.  The stencil rows
// live in a shared-memory ring of ROWS + 2R + 1 rows, so a band copies in
// only its ROWS new rows.  Thread (lane, w) of a band computes the y face
// (i, j+1/2) and the x face (i+1/2, j) of point (i, j), j = j0 + w: the y
// fluxes go to a shared buffer of ROWS + 1 face rows (a band's bottom faces
// are the previous band's top faces; the first band of a segment starts one
// row lower, where warp 0 computes the segment's bottom faces), the x flux of
// i-1/2 comes by warp shuffle, and the point is
// updated as in k_xupd.  Against k_yface + k_xupd the y fluxes never leave
// the SM, every stencil value is copied in once per stage, and the velocity
// reconstructions that the superluminal fall-back of HLL / HLLC couples
// between the two faces of a point are formed once.
constexpr int NF_RING = 21;   // 0-4 time-n vx, vy, vz, p, rho; 5-18 stage psi .. Sz; 19 Jx; 20 Jy

template <int RM, int ROWS>
struct RingGeom {
  static constexpr int R = MPR<RM>::R;
  static constexpr int NS = 2 * R + 2;
  static constexpr int NR = ROWS + 2 * R + 1;          // ring rows
  // staged columns: cs .. cs + LONG - 1 with cs = (i0 - R) rounded down to
  // an even column (16-byte aligned rows for the bulk copies), covering the
  // stencils' i0-R .. i0+32+R
  static constexpr int LONG = 32 + 2 * R + 2;
  static constexpr int ROWSZ = NF_RING * LONG;         // doubles per ring row
  static constexpr int RING = NR * ROWSZ;
  static constexpr int YF = (ROWS + 1) * NROLE * 32;   // y-flux face rows x roles x lanes
  static constexpr size_t bytes() { return sizeof(double) * (size_t)(RING + YF); }
  // ring row of grid row r (r > -16 NR)
  static __device__ __forceinline__ int slot(int r) { return (int)((unsigned)(r + 16 * NR) % (unsigned)NR); }
};
// the fused kernel is built where two CTAs of FACE_ROWS warps fit an SM's
// 228 KB of shared memory (MP5 and the MC slopes)
template <int RM>
constexpr bool kFused = RingGeom<RM, FACE_ROWS>::bytes() <= 113 * 1024;

// first staged column of a strip (see RingGeom::LONG)
template <int R>
__device__ __forceinline__ int ring_col0(int i0) { return (i0 - R) & ~1; }

// Whether a strip's staged columns are all interior points: then every ring
// row is one contiguous, 16-byte aligned segment of LONG doubles per field
// (rows outside 0..jmax map to interior rows), copied by the bulk-copy
// engine; strips at the x boundaries go element by element through the
// ghost map.
template <int RM, int ROWS>
__device__ __forceinline__ bool ring_bulk(const InstDesc& I, int i0) {
  const int cs = ring_col0<MPR<RM>::R>(i0);
  return cs >= 0 && cs + RingGeom<RM, ROWS>::LONG - 1 <= I.imax;
}

// staged field f (0-4 time-n vx, vy, vz, p, rho; 5-20 stage psi .. Sz, Jx, Jy)
__device__ __forceinline__ const double* ring_field(const double* prim, const double* Q, long long fs, int f) {
  if (f < 5) return prim + (long long)(f < 3 ? P_VX + f : (f == 3 ? P_P : P_RHO)) * fs;
  return Q + (long long)(f - 5) * fs;
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(umma::smem_u32(bar)), "r"(bytes)
               : "memory");
}
// one bulk copy global -> shared of `bytes` (16-byte aligned addresses, a
// multiple of 16 bytes) completing on the CTA's mbarrier `bar`
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   umma::smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(umma::smem_u32(bar))
               : "memory");
}

// copies grid rows ra .. rb of the strip into their ring rows: with bulk,
// one bulk copy per field and row, spread over all the CTA's threads
// (completion on bar, which the caller waits for), else element by element
// through the ghost maps
// (columns i0-R .. ilast+R+1; the caller waits with cp.async.wait_all)
template <int RM, int ROWS>
__device__ __forceinline__ void ring_fill(const InstDesc& I, const StageArgs& sa, double* ring, int i0, int ilast,
                                          int ra, int rb, int tid, bool bulk, uint64_t* bar) {
  using G = RingGeom<RM, ROWS>;
  constexpr int R = G::R, LONG = G::LONG;
  const long long fs = I.fstride;
  const double* __restrict__ prim = I.prim[sa.cur];
  const double* __restrict__ Q = I.stage[sa.qin];
  const int cs = ring_col0<R>(i0);
  if (bulk) {
    // every thread arrives once per fill (the barrier counts all of them),
    // announcing the bytes of the copies it issues itself
    const int n = (rb - ra + 1) * NF_RING;
    constexpr uint32_t kRowBytes = LONG * sizeof(double);
    uint32_t mine = 0;
    for (int e = tid; e < n; e += 32 * ROWS) mine += kRowBytes;
    // the ring rows being replaced were read through the generic proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_arrive_expect_tx(bar, mine);
    for (int e = tid; e < n; e += 32 * ROWS) {
      const int r = e / NF_RING, f = e - r * NF_RING, row = ra + r;
      const double* src = ring_field(prim, Q, fs, f) + (long long)map_idx(row, I.jmax, I.bc_y) * I.pitch + cs;
      bulk_g2s(ring + G::slot(row) * G::ROWSZ + f * LONG, src, kRowBytes, bar);
    }
    return;
  }
  const int cfirst = i0 - R - cs, clast = ilast + R + 1 - cs;   // needed ring columns
  const int n = (rb - ra + 1) * LONG;
  for (int e = tid; e < n; e += 32 * ROWS) {
    const int r = e / LONG, c = e - r * LONG;
    if (c < cfirst || c > clast) continue;
    const int row = ra + r;
    const long long off = (long long)map_idx(row, I.jmax, I.bc_y) * I.pitch + map_idx(cs + c, I.imax, I.bc_x);
    double* dst = ring + G::slot(row) * G::ROWSZ + c;
    cp_async8(dst + 0 * LONG, prim + P_VX * fs + off);
    cp_async8(dst + 1 * LONG, prim + P_VY * fs + off);
    cp_async8(dst + 2 * LONG, prim + P_VZ * fs + off);
    cp_async8(dst + 3 * LONG, prim + P_P * fs + off);
    cp_async8(dst + 4 * LONG, prim + P_RHO * fs + off);
#pragma unroll
    for (int f = 0; f < 16; ++f) cp_async8(dst + (5 + f) * LONG, Q + f * fs + off);   // psi .. Sz, Jx, Jy
  }
}

// stencil values of the face of (i, j) in direction D from the ring:
// D = 0 row j, columns i-R .. i+R+1; D = 1 column i, rows j-R .. j+R+1
template <int RM, int ROWS, int D>
struct RingAcc {
  using G = RingGeom<RM, ROWS>;
  const double* ring;
  int off[D == 0 ? 1 : G::NS];
  __device__ __forceinline__ double n(int f, int q) const {
    const int ff = (D == 1 && f == 19) ? 20 : f;   // field 19 is the normal current
    if constexpr (D == 0) return ring[off[0] + ff * G::LONG + q];
    else return ring[off[q] + ff * G::LONG];
  }
  __device__ __forceinline__ double t(int, int) const { return 0.0; }   // the fused faces take FacePre
};

template <int RM, typename T, bool POS, class ACC>
__device__ __forceinline__ Pair<T> rec_acc(const ACC& a, int f) {
  constexpr int NS = 2 * MPR<RM>::R + 2;
  T u[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) u[q] = T(a.n(f, q));
  return MPCall<RM, T>::template call<POS>(u);
}

// pressure face values of one direction (positivity-fixed pair; the
// split-pressure solvers reconstruct differences from the face cell's value)
template <int RM, int SOLVER, typename T, class ACC>
__device__ __forceinline__ void pressure_pair(const ACC& a, FacePre<T>& pre) {
  if constexpr (kSplitP<T, SOLVER>) {
    constexpr int R = MPR<RM>::R, NS = 2 * R + 2;
    const double c0 = a.n(3, R);
    T u[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) u[q] = T(a.n(3, q) - c0);
    const Pair<T> pp = MPCall<RM, T>::call_posd(u, c0);
    pre.pc0 = c0;
    pre.dpL = pp.L; pre.dpR = pp.R;
    pre.pL = T(c0 + double(pp.L)); pre.pR = T(c0 + double(pp.R));
  } else {
    const Pair<T> pp = rec_acc<RM, T, true>(a, 3);
    pre.pL = pp.L; pre.pR = pp.R;
  }
}

// velocity slots of both faces of point (i, j) with the superluminal
// fall-back of 16_hll_flow_mpx.f95:1393-1462: if any of the four
// reconstructions is superluminal, both faces take cell (i, j) on the left
// and cell (i-1, j) (x) or (i, j-1) (y) on the right
template <int RM, typename T, class AX, class AY>
__device__ __forceinline__ void point_velocities(const AX& ax, const AY& ay, T (&xL)[3], T (&xR)[3], T (&yL)[3],
                                                 T (&yR)[3]) {
  constexpr int R = MPR<RM>::R;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const Pair<T> px = rec_acc<RM, T, false>(ax, c);
    xL[c] = px.L; xR[c] = px.R;
    const Pair<T> py = rec_acc<RM, T, false>(ay, c);
    yL[c] = py.L; yR[c] = py.R;
  }
  const T V2xl = pw2(xL[0]) + pw2(xL[1]) + pw2(xL[2]);
  const T V2xr = pw2(xR[0]) + pw2(xR[1]) + pw2(xR[2]);
  const T V2yl = pw2(yL[0]) + pw2(yL[1]) + pw2(yL[2]);
  const T V2yr = pw2(yR[0]) + pw2(yR[1]) + pw2(yR[2]);
  if (V2xl >= T(1) || V2xr >= T(1) || V2yl >= T(1) || V2yr >= T(1)) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      xL[c] = T(ax.n(c, R)); xR[c] = T(ax.n(c, R - 1));
      yL[c] = T(ay.n(c, R)); yR[c] = T(ay.n(c, R - 1));
    }
  }
}

// y face (i, j+1/2) of point (i, j).  For HLL / HLLC the point's x-face
// velocity slots are parked in xstash (6 doubles, stride 32: shared memory
// that the caller reloads before it stores the y fluxes there) and yneg tells
// whether a raw y density face value is negative (the x density fix-up of
// 16_hllc_flow_mpx.f95:2663-2690 looks at the y pair first)
template <int RM, int SOLVER, typename T, int ROWS>
__device__ __forceinline__ uint32_t fused_yface(const RingAcc<RM, ROWS, 0>& ax, const RingAcc<RM, ROWS, 1>& ay,
                                                const InstDesc& I, volatile double* xstash, bool& yneg,
                                                flux_t<T, SOLVER> (&F)[NROLE]) {
  constexpr int R = MPR<RM>::R;
  yneg = false;
  if constexpr (SOLVER == 5 || SOLVER == 7) {
    FacePre<T> py;
    {
      T xL[3], xR[3];
      point_velocities<RM, T>(ax, ay, xL, xR, py.vL, py.vR);
      if (xstash) {
#pragma unroll
        for (int c = 0; c < 3; ++c) { xstash[c * 32] = double(xL[c]); xstash[(3 + c) * 32] = double(xR[c]); }
      }
    }
    pressure_pair<RM, SOLVER, T>(ay, py);
    const Pair<T> pr = rec_acc<RM, T, true>(ay, 4);
    py.rhoL = pr.L; py.rhoR = pr.R;
    if constexpr (SOLVER == 7) {
      yneg = (py.rhoL < T(0)) || (py.rhoR < T(0));
      if (yneg) {
        const T r10 = T(ay.n(4, R) * 1.0e-1);
        if (py.rhoL < T(0)) py.rhoL = r10;
        else py.rhoR = r10;
      }
    }
    return face_flux<RM, SOLVER, T, 1, true>(ay, &py, I.gamma, I.sigma, F);
  } else {
    return face_flux<RM, SOLVER, T, 1, false>(ay, (const FacePre<T>*)nullptr, I.gamma, I.sigma, F);
  }
}

// x face (i+1/2, j) of point (i, j); xv = the velocity slots fused_yface parked
template <int RM, int SOLVER, typename T, int ROWS>
__device__ __forceinline__ uint32_t fused_xface(const RingAcc<RM, ROWS, 0>& ax, const InstDesc& I, const T (&xv)[6],
                                                bool yneg, flux_t<T, SOLVER> (&F)[NROLE]) {
  constexpr int R = MPR<RM>::R;
  if constexpr (SOLVER == 5 || SOLVER == 7) {
    FacePre<T> px;
#pragma unroll
    for (int c = 0; c < 3; ++c) { px.vL[c] = xv[c]; px.vR[c] = xv[3 + c]; }
    pressure_pair<RM, SOLVER, T>(ax, px);
    const Pair<T> pr = rec_acc<RM, T, true>(ax, 4);
    px.rhoL = pr.L; px.rhoR = pr.R;
    if constexpr (SOLVER == 7) {
      if ((px.rhoL < T(0) || px.rhoR < T(0)) && !yneg) {
        const T r10 = T(ax.n(4, R) * 1.0e-1);
        if (px.rhoL < T(0)) px.rhoL = r10;
        else px.rhoR = r10;
      }
    }
    return face_flux<RM, SOLVER, T, 0, true>(ax, &px, I.gamma, I.sigma, F);
  } else {
    return face_flux<RM, SOLVER, T, 0, false>(ax, (const FacePre<T>*)nullptr, I.gamma, I.sigma, F);
  }
}

template <int RM, int SOLVER, typename T, int EP, int ROWS>
__global__ void __launch_bounds__(32 * ROWS, 16 / ROWS)
k_stage(const InstDesc* __restrict__ insts, int ninst, int ntiles, StageArgs sa) {
  using G = RingGeom<RM, ROWS>;
  constexpr int R = G::R, NS = G::NS, LONG = G::LONG;
  constexpr bool kPre = SOLVER == 5 || SOLVER == 7;
  extern __shared__ __align__(128) double smem[];
  __shared__ __align__(8) uint64_t bar;   // completion of the bulk copies of a band's rows
  double* ring = smem;
  double* yf = smem + G::RING;
  const int lane = threadIdx.x, w = threadIdx.y, tid = w * 32 + lane;
  if (tid == 0) {
    umma::mbar_init(&bar, 32 * ROWS);   // every thread arrives once per bulk fill
    umma::mbar_fence_init();
  }
  __syncthreads();
  uint32_t bulk_phase = 0;   // parity of the next bulk fill to complete
  constexpr uint32_t kCopyPolls = 1u << 22;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int b = tile;
    const InstDesc& I = tile_inst(insts, ninst, LK_STAGE, b);
    const int nstrip = (I.imax + 1 + 30) / 31;
    const int i0 = (b % nstrip) * 31 - 1, jseg = (b / nstrip) * I.seg_rows;
    const int ilast = min(i0 + 31, I.imax), jend = min(jseg + I.seg_rows - 1, I.jmax);
    const int i = i0 + lane;
    const bool bulk = ring_bulk<RM, ROWS>(I, i0);
    const int sh = i0 - R - ring_col0<R>(i0);   // ring column of grid column i0 - R (0 or 1)
    uint32_t stt = 0;
    auto x_acc = [&](int j) {
      RingAcc<RM, ROWS, 0> a{ring, {G::slot(j) * G::ROWSZ + lane + sh}};
      return a;
    };
    auto y_acc = [&](int j) {
      RingAcc<RM, ROWS, 1> a;
      a.ring = ring;
#pragma unroll
      for (int q = 0; q < NS; ++q) a.off[q] = G::slot(j - R + q) * G::ROWSZ + lane + R + sh;
      return a;
    };
    // The bands start one row below the segment: warp 0 of the first band
    // computes only the y faces jseg - 1/2 (the segment's bottom faces; row
    // jseg - 1 belongs to the segment below and is not updated here), every
    // other warp the y face, the x face and the update of its row.  With
    // seg_rows = 8 nb - 1 the bands are full.
    const int jfirst = jseg - 1;
    ring_fill<RM, ROWS>(I, sa, ring, i0, ilast, jfirst - R, min(jfirst + ROWS - 1, jend) + R + 1, tid, bulk, &bar);
    int band = 0;
    for (int j0 = jfirst; j0 <= jend; j0 += ROWS, ++band) {
      const int jl = min(j0 + ROWS - 1, jend);
      if constexpr (EP != EP_RHS) prefetch_update_rows(I, sa, i0, ilast, max(j0, jseg), jl, tid, 32 * ROWS);
      // the band's rows have arrived, and every warp has finished the previous
      // band's update (its reads of the face rows that this band overwrites)
      if (bulk) {
        const bool ok = umma::mbar_wait(&bar, bulk_phase, kCopyPolls);
        if (!__syncthreads_and(ok)) {
          // the copies did not arrive in time: report, wait (bounded) for the
          // ones still in flight, and stop the CTA
          if (tid == 0) {
            atomicOr(I.status, ST_COPY_TIMEOUT);
            umma::mbar_wait(&bar, bulk_phase, kCopyPolls);
          }
          __syncthreads();
          return;
        }
        bulk_phase ^= 1u;
      } else {
        cp_async_wait_all();
        __syncthreads();
      }
      // face row k of this band (k = 0 bottom faces, k = w + 1 the faces above row w)
      const int rb = (band * ROWS) % (ROWS + 1);
      auto frow = [&](int k) { const int r = k + rb; return yf + (r >= ROWS + 1 ? r - (ROWS + 1) : r) * (NROLE * 32); };
      const int j = j0 + w;
      const bool face_only = j < jseg;   // warp 0 of the first band
      const bool valid = lane >= 1 && i <= ilast;
      const bool warp_c2p = EP == EP_LAST && I.c2p == 2 && !I.c2p_tc;
      // point whose update this lane computes (lanes without one repeat a real
      // point in the warp-wide con2prim, and store nothing)
      const int ii = valid ? i : (lane == 0 ? i0 + 1 : ilast);
      const int ln = ii - i0;
      flux_t<T, SOLVER> Fx[NROLE];
#pragma unroll
      for (int c = 0; c < NROLE; ++c) Fx[c] = 0;
      Centre cv{};
      if (j <= jl) {
        if (i <= ilast) {
          const RingAcc<RM, ROWS, 0> ax = x_acc(j);
          volatile double* top = frow(w + 1) + lane;
          bool yneg;
          T xv[6];
          {
            flux_t<T, SOLVER> Fy[NROLE];
            stt |= fused_yface<RM, SOLVER, T, ROWS>(ax, y_acc(j), I, kPre ? top : nullptr, yneg, Fy);
            if constexpr (kPre) {
#pragma unroll
              for (int c = 0; c < 6; ++c) xv[c] = T(top[c * 32]);
            }
#pragma unroll
            for (int c = 0; c < NROLE; ++c) top[c * 32] = double(Fy[c]);
          }
          if (!face_only) stt |= fused_xface<RM, SOLVER, T, ROWS>(ax, I, xv, yneg, Fx);
        }
        // centre values of the point, read before the next band's copies
        // replace the ring rows
        const double* cen = ring + G::slot(j) * G::ROWSZ + ln + R + sh;
        auto cs = [&](int f) { return cen[f * LONG]; };
        cv = Centre{cs(5 + Q_Q), cs(5 + Q_PSI), cs(5 + Q_PHI), cs(5 + Q_EX), cs(5 + Q_EY), cs(5 + Q_EZ),
                    cs(5 + Q_BX), cs(5 + Q_BY), cs(5 + Q_BZ), cs(0), cs(1), cs(2)};
      }
      __syncthreads();   // the band's y fluxes are complete and its ring reads done
      if (j0 + ROWS <= jend)   // the next band's rows arrive while this band updates
        ring_fill<RM, ROWS>(I, sa, ring, i0, ilast, j0 + ROWS + R + 1, min(j0 + 2 * ROWS - 1, jend) + R + 1, tid,
                            bulk, &bar);
      if (j <= jl && !face_only) {
        const double dlx = I.delx, ix2 = I.inv_delx_pow2;
        double qx[NROLE];
#pragma unroll
        for (int c = 0; c < NROLE; ++c) {
          const double fr = double(Fx[c]);
          const double fl = __shfl_up_sync(0xffffffffu, fr, 1);
          const double d = fr - fl;
          qx[c] = ix2 != 0.0 ? d * ix2 : d / dlx;
        }
        if (valid || warp_c2p) {
          if (warp_c2p) {
#pragma unroll
            for (int c = 0; c < NROLE; ++c) qx[c] = __shfl_sync(0xffffffffu, qx[c], ln);
          }
          const double* ytop = frow(w + 1) + ln;
          const double* ybot = frow(w) + ln;
          auto fyd = [&](int r) { return ytop[r * 32] - ybot[r * 32]; };
          stt |= update_point<EP, T, SOLVER>(I, sa, ii, j, qx, fyd, cv, valid);
        }
      }
    }
    __syncthreads();   // the next tile's copies overwrite the ring and the face rows
    if (stt) atomicOr(I.status, stt);
  }
}

// ---------------------------------------------------------------- launchers
template <int RM, int SV, typename T, int ROWS>
static void launch_tiles(const StageShape& sh, cudaStream_t st, const InstDesc* d, int n, const StageArgs& sa,
                         cudaEvent_t* ev) {
  using G = FaceGeom<RM, SV, ROWS>;
  const dim3 blk(32, ROWS);
  if constexpr (kFused<RM> && ROWS == FACE_ROWS) {
    if (sh.fused && sa.mode == 0) {
      // one launch: ev[0] and ev[1] bracket no work (no separate y-face kernel)
      using RG = RingGeom<RM, ROWS>;
      if (ev) { cudaEventRecord(ev[0], st); cudaEventRecord(ev[1], st); }
      const int gs = sh.grid[LK_STAGE], ns = sh.ntiles[LK_STAGE];
      if (sa.l < sa.s) k_stage<RM, SV, T, EP_MID, ROWS><<<gs, blk, RG::bytes(), st>>>(d, n, ns, sa);
      else k_stage<RM, SV, T, EP_LAST, ROWS><<<gs, blk, RG::bytes(), st>>>(d, n, ns, sa);
      if (ev) cudaEventRecord(ev[2], st);
      return;
    }
  }
  if (ev) cudaEventRecord(ev[0], st);
  k_yface<RM, SV, T, ROWS><<<sh.grid[LK_YFACE], blk, G::bytes(1), st>>>(d, n, sh.ntiles[LK_YFACE], sa);
  if (ev) cudaEventRecord(ev[1], st);
  const int gx = sh.grid[LK_XUPD], nt = sh.ntiles[LK_XUPD];
  if (sa.mode >= 1) k_xupd<RM, SV, T, EP_RHS, ROWS><<<gx, blk, G::bytes(0), st>>>(d, n, nt, sa);
  else if (sa.l < sa.s) k_xupd<RM, SV, T, EP_MID, ROWS><<<gx, blk, G::bytes(0), st>>>(d, n, nt, sa);
  else k_xupd<RM, SV, T, EP_LAST, ROWS><<<gx, blk, G::bytes(0), st>>>(d, n, nt, sa);
  if (ev) cudaEventRecord(ev[2], st);
}

template <int RM, int SV, typename T, int ROWS>
static cudaError_t prepare_tiles() {
  using G = FaceGeom<RM, SV, ROWS>;
  const int b0 = (int)G::bytes(0), b1 = (int)G::bytes(1);
  cudaError_t e = cudaFuncSetAttribute(k_yface<RM, SV, T, ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize, b1);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_xupd<RM, SV, T, EP_RHS, ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize, b0);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_xupd<RM, SV, T, EP_MID, ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize, b0);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_xupd<RM, SV, T, EP_LAST, ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize, b0);
  if constexpr (kFused<RM> && ROWS == FACE_ROWS) {
    const int bs = (int)RingGeom<RM, ROWS>::bytes();
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_stage<RM, SV, T, EP_MID, ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bs);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_stage<RM, SV, T, EP_LAST, ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bs);
  }
  return e;
}

template <int RM, int SV, typename T>
static void launch_rm_sv(const StageShape& sh, cudaStream_t st, const InstDesc* d, int n, const StageArgs& sa,
                         cudaEvent_t* ev) {
  if (sh.rows == 4) launch_tiles<RM, SV, T, 4>(sh, st, d, n, sa, ev);
  else launch_tiles<RM, SV, T, 8>(sh, st, d, n, sa, ev);
}

template <int RM, int SV, typename T>
static cudaError_t prepare_rm_sv() {
  cudaError_t e = prepare_tiles<RM, SV, T, 8>();
  if (e == cudaSuccess) e = prepare_tiles<RM, SV, T, 4>();
  return e;
}

// one solver's stage launch / kernel set-up over rec_mp in one precision
// (T = double: plain FP64; T = float: the mixed-precision kernels, which the
// build compiles in translation units of their own)
template <int SV, typename T>
cudaError_t launch_stage_solver(int rec_mp, const StageShape& sh, cudaStream_t st, const InstDesc* d, int n,
                                const StageArgs& sa, cudaEvent_t* ev) {
  if (sh.rows != 4 && sh.rows != 8) return cudaErrorInvalidValue;
  if constexpr (SV >= 1 && SV <= 4) {   // the MC family uses MC slopes; rec_mp does not apply
    launch_rm_sv<3, SV, T>(sh, st, d, n, sa, ev);
  } else {
    switch (rec_mp) {
      case 0: launch_rm_sv<0, SV, T>(sh, st, d, n, sa, ev); break;
      case 1: launch_rm_sv<1, SV, T>(sh, st, d, n, sa, ev); break;
      case 2: launch_rm_sv<2, SV, T>(sh, st, d, n, sa, ev); break;
      default: return cudaErrorInvalidValue;
    }
  }
  return cudaGetLastError();
}

template <int SV, typename T>
cudaError_t prepare_stage_solver(int rec_mp) {
  if constexpr (SV >= 1 && SV <= 4) {
    return prepare_rm_sv<3, SV, T>();
  } else {
    switch (rec_mp) {
      case 0: return prepare_rm_sv<0, SV, T>();
      case 1: return prepare_rm_sv<1, SV, T>();
      case 2: return prepare_rm_sv<2, SV, T>();
      default: return cudaErrorInvalidValue;
    }
  }
}

// A solver's translation unit defines its launcher and set-up for one
// precision: compiled plain for FP64 (<name>_fp64), or with
// CUEVA_STAGE_MIXED for the mixed-precision kernels (<name>_mixed).
#if defined(CUEVA_STAGE_MIXED)
#define CUEVA_STAGE_UNIT(NAME, SV)                                                                              \
  cudaError_t launch_stage_##NAME##_mixed(int rec_mp, const StageShape& sh, cudaStream_t st, const InstDesc* d, \
                                          int n, const StageArgs& sa, cudaEvent_t* ev) {                       \
    return launch_stage_solver<SV, float>(rec_mp, sh, st, d, n, sa, ev);                                       \
  }                                                                                                            \
  cudaError_t prepare_stage_##NAME##_mixed(int rec_mp) { return prepare_stage_solver<SV, float>(rec_mp); }
#else
#define CUEVA_STAGE_UNIT(NAME, SV)                                                                             \
  cudaError_t launch_stage_##NAME##_fp64(int rec_mp, const StageShape& sh, cudaStream_t st, const InstDesc* d, \
                                         int n, const StageArgs& sa, cudaEvent_t* ev) {                       \
    return launch_stage_solver<SV, double>(rec_mp, sh, st, d, n, sa, ev);                                     \
  }                                                                                                           \
  cudaError_t prepare_stage_##NAME##_fp64(int rec_mp) { return prepare_stage_solver<SV, double>(rec_mp); }
#endif

}  // namespace cueva
