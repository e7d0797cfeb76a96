// cueva_riemann.cuh -- per-interface HLL / HLLC fluxes of the resistive RMHD
// system, one direction at a time.
//
// Reference: 16_hll_flow_mpx.f95:1358-1965 (HLL) and
// 16_hllc_flow_mpx.f95:2401-4618 (HLLC).  The Fortran writes the x and y
// branches out separately; they are the same formulas under the cyclic map
// (x,y,z) -> (y,z,x), so one direction template serves both.  Components are
// addressed by role: n (normal), t1, t2 with (n,t1,t2) = (x,y,z) for the x
// interfaces and (y,z,x) for the y interfaces.  The only place where the
// Fortran does not follow the cyclic map is the y-interface momentum flux
// FSyx = ... + h W^2 vx vy (x first), handled below.  Isotropic sums
// (|v|^2, |E|^2+|B|^2) keep the Fortran x,y,z order in both directions.
//
// The Fortran reconstructs -E and -B as separate slots (16_hll_flow_mpx.f95:
// 791-801); MP5/7/9 are exactly odd-symmetric in IEEE arithmetic, so those
// slots are the negated E and B values and the formulas below use the
// negation directly (identical values, zero signs aside).
//
// Output: 14 interface fluxes in role order (see enum Role).  The divergence
// (17_fluxandsource.f95) consumes them with the reference's array signs:
//   R_BT1 holds EzlaxBy (x) / ExlaxBz (y)    = -F(B_t1)
//   R_ET2 holds BylaxEz (x) / BzlaxEx (y)    = -F(E_t2)
//   all other roles hold the flux itself.
#pragma once
#include "cueva_common.cuh"

namespace cueva {

enum Role { R_PSI = 0, R_PHI, R_BN, R_BT1, R_BT2, R_EN, R_ET1, R_ET2, R_Q, R_D, R_TAU, R_SN, R_ST1, R_ST2, NROLE };
static_assert(NROLE == NFACE, "flux scratch holds one slab per role");

template <typename T>
struct Side {
  T psi, phi, Ex, Ey, Ez, Bx, By, Bz, q, D, tau, Sx, Sy, Sz, vx, vy, vz, p, rho, J;
};

// role accessors
template <int D> struct Dir;
template <> struct Dir<0> {
  template <class S> static __device__ __forceinline__ auto En(const S& s) { return s.Ex; }
  template <class S> static __device__ __forceinline__ auto Et1(const S& s) { return s.Ey; }
  template <class S> static __device__ __forceinline__ auto Et2(const S& s) { return s.Ez; }
  template <class S> static __device__ __forceinline__ auto Bn(const S& s) { return s.Bx; }
  template <class S> static __device__ __forceinline__ auto Bt1(const S& s) { return s.By; }
  template <class S> static __device__ __forceinline__ auto Bt2(const S& s) { return s.Bz; }
  template <class S> static __device__ __forceinline__ auto Sn(const S& s) { return s.Sx; }
  template <class S> static __device__ __forceinline__ auto St1(const S& s) { return s.Sy; }
  template <class S> static __device__ __forceinline__ auto St2(const S& s) { return s.Sz; }
  template <class S> static __device__ __forceinline__ auto vn(const S& s) { return s.vx; }
  template <class S> static __device__ __forceinline__ auto vt1(const S& s) { return s.vy; }
  template <class S> static __device__ __forceinline__ auto vt2(const S& s) { return s.vz; }
};
template <> struct Dir<1> {
  template <class S> static __device__ __forceinline__ auto En(const S& s) { return s.Ey; }
  template <class S> static __device__ __forceinline__ auto Et1(const S& s) { return s.Ez; }
  template <class S> static __device__ __forceinline__ auto Et2(const S& s) { return s.Ex; }
  template <class S> static __device__ __forceinline__ auto Bn(const S& s) { return s.By; }
  template <class S> static __device__ __forceinline__ auto Bt1(const S& s) { return s.Bz; }
  template <class S> static __device__ __forceinline__ auto Bt2(const S& s) { return s.Bx; }
  template <class S> static __device__ __forceinline__ auto Sn(const S& s) { return s.Sy; }
  template <class S> static __device__ __forceinline__ auto St1(const S& s) { return s.Sz; }
  template <class S> static __device__ __forceinline__ auto St2(const S& s) { return s.Sx; }
  template <class S> static __device__ __forceinline__ auto vn(const S& s) { return s.vy; }
  template <class S> static __device__ __forceinline__ auto vt1(const S& s) { return s.vz; }
  template <class S> static __device__ __forceinline__ auto vt2(const S& s) { return s.vx; }
};

// physical fluxes of one reconstructed side, 16_hll_flow_mpx.f95:1464-1733
template <typename T> struct Phys { T FD, Ftau, FSn, FSt1, FSt2; };

template <int D, typename T>
__device__ __forceinline__ Phys<T> physical(const Side<T>& s, T gamma) {
  using X = Dir<D>;
  Phys<T> f;
  const T V2 = pw2(s.vx) + pw2(s.vy) + pw2(s.vz);
  const T W = T(1.0) / sqrt(T(1.0) - V2);
  const T E2B2 = pw2(s.Ex) + pw2(s.Ey) + pw2(s.Ez) + pw2(s.Bx) + pw2(s.By) + pw2(s.Bz);
  const T eps = s.p / ((gamma - T(1.0)) * s.rho);
  const T h = s.rho * (T(1.0) + eps) + s.p;
  const T hW2 = h * pw2(W);
  const T vn = X::vn(s), vt1 = X::vt1(s), vt2 = X::vt2(s);
  const T En = X::En(s), Et1 = X::Et1(s), Et2 = X::Et2(s);
  const T Bn = X::Bn(s), Bt1 = X::Bt1(s), Bt2 = X::Bt2(s);
  f.FD = s.D * vn;
  f.Ftau = (Bt2 * Et1 - Bt1 * Et2) + hW2 * vn;
  f.FSn = -pw2(En) - pw2(Bn) + hW2 * pw2(vn) + T(0.5) * E2B2 + s.p;
  f.FSt1 = -En * Et1 - Bn * Bt1 + hW2 * vn * vt1;
  if constexpr (D == 0) f.FSt2 = -En * Et2 - Bn * Bt2 + hW2 * vn * vt2;
  else                  f.FSt2 = -En * Et2 - Bn * Bt2 + hW2 * vt2 * vn;   // FSyx: vx before vy
  return f;
}

// fixed-speed (s1 = -1, s2 = +1) HLL combination
// (s2*FL - s1*FR + s1*s2*(UR-UL))/(s2-s1) == 0.5*((FL+FR) - (UR-UL)) exactly
template <typename T>
__device__ __forceinline__ T hll(T FL, T FR, T UL, T UR) { return T(0.5) * ((FL + FR) - (UR - UL)); }

// EM and charge fluxes (identical for HLL, HLLC and the HLLE EM part)
template <int D, typename T>
__device__ __forceinline__ void em_fluxes(const Side<T>& L, const Side<T>& R, T* A) {
  using X = Dir<D>;
  A[R_PSI] = hll(X::En(L), X::En(R), L.psi, R.psi);
  A[R_PHI] = hll(X::Bn(L), X::Bn(R), L.phi, R.phi);
  A[R_BN] = hll(L.phi, R.phi, X::Bn(L), X::Bn(R));
  A[R_BT1] = T(0.5) * ((X::Et2(L) + X::Et2(R)) + (X::Bt1(R) - X::Bt1(L)));
  A[R_BT2] = hll(X::Et1(L), X::Et1(R), X::Bt2(L), X::Bt2(R));
  A[R_EN] = hll(L.psi, R.psi, X::En(L), X::En(R));
  A[R_ET1] = hll(X::Bt2(L), X::Bt2(R), X::Et1(L), X::Et1(R));
  A[R_ET2] = T(0.5) * ((X::Bt1(L) + X::Bt1(R)) + (X::Et2(R) - X::Et2(L)));
  A[R_Q] = hll(L.J, R.J, L.q, R.q);
}

template <int D, typename T>
__device__ __forceinline__ void hll_fluxes(const Side<T>& L, const Side<T>& R, T gamma, T* A) {
  using X = Dir<D>;
  em_fluxes<D>(L, R, A);
  const Phys<T> fl = physical<D>(L, gamma), fr = physical<D>(R, gamma);
  A[R_D] = hll(fl.FD, fr.FD, L.D, R.D);
  A[R_TAU] = hll(fl.Ftau, fr.Ftau, L.tau, R.tau);
  A[R_SN] = hll(fl.FSn, fr.FSn, X::Sn(L), X::Sn(R));
  A[R_ST1] = hll(fl.FSt1, fr.FSt1, X::St1(L), X::St1(R));
  A[R_ST2] = hll(fl.FSt2, fr.FSt2, X::St2(L), X::St2(R));
}

// get_hllc_vel, funciones.f95:188-259: Newton on a v^2 - b v + c = 0 in
// [-1,1].  The Fortran's first f evaluation reads the local v before it is
// assigned (line 229); this evaluates it at the seed oldv, like the oracle.
// The reference's step tolerance 1e-12 is below FP32 resolution, so the FP32
// (mixed-precision) instantiation stops at 4e-7, two ulps of |v| <= 1.
template <typename T>
__device__ __forceinline__ T hllc_vel(T a, T b, T c, T rt, uint32_t& st) {
  const T tol = (sizeof(T) == sizeof(double)) ? T(1.0e-12) : T(4.0e-7);
  T oldv = fmax2(T(-1.0), fmin2(T(1.0), rt));
  T v = oldv;
  for (int iter = 1;; ++iter) {
    const T fv = a * v * v - b * v + c;
    const T dfdv = T(2.0) * a * v - b;
    v = fmax2(T(-1.0), fmin2(T(1.0), oldv - fv / dfdv));
    const T err = fabs(oldv - v);
    oldv = v;
    if (iter >= 100) { st |= ST_HLLC_NOCONV; break; }
    if (!(err > tol)) break;
  }
  return fmax2(T(-1.0) + T(1.0e-3), fmin2(T(1.0) - T(1.0e-3), v));
}

// HLLC of Miranda-Aranguren et al. (2018), 16_hllc_flow_mpx.f95:2816-4610
template <int D, typename T>
__device__ __forceinline__ void hllc_fluxes(const Side<T>& L, const Side<T>& R, T gamma, T* A, uint32_t& st) {
  using X = Dir<D>;
  em_fluxes<D>(L, R, A);
  const Phys<T> fl = physical<D>(L, gamma), fr = physical<D>(R, gamma);
  const T h = T(0.5);
  // HLL averages of the state (:2816-2900)
  const T psi_hll = h * (((R.psi + L.psi) + X::En(L)) - X::En(R));
  const T phi_hll = h * (((R.phi + L.phi) + X::Bn(L)) - X::Bn(R));
  const T En_hll = h * (((X::En(R) + X::En(L)) + L.psi) - R.psi);
  const T Et1_hll = h * (((X::Et1(R) + X::Et1(L)) + X::Bt2(L)) - X::Bt2(R));
  const T Et2_hll = h * (((X::Et2(R) + X::Et2(L)) - X::Bt1(L)) + X::Bt1(R));
  const T Bn_hll = h * (((X::Bn(R) + X::Bn(L)) + L.phi) - R.phi);
  const T Bt1_hll = h * (((X::Bt1(R) + X::Bt1(L)) - X::Et2(L)) + X::Et2(R));
  const T Bt2_hll = h * (((X::Bt2(R) + X::Bt2(L)) + X::Et1(L)) - X::Et1(R));
  const T D_hll = h * (((R.D + L.D) + fl.FD) - fr.FD);
  const T tau_hll = h * (((R.tau + L.tau) + fl.Ftau) - fr.Ftau);
  const T Sn_hll = h * (((X::Sn(R) + X::Sn(L)) + fl.FSn) - fr.FSn);
  const T St1_hll = h * (((X::St1(R) + X::St1(L)) + fl.FSt1) - fr.FSt1);
  const T St2_hll = h * (((X::St2(R) + X::St2(L)) + fl.FSt2) - fr.FSt2);
  // HLL fluxes that enter the star states (:2904-3100)
  const T psi_f = A[R_PSI];
  const T phi_f = A[R_PHI];
  const T En_f = A[R_EN];
  const T Bn_f = A[R_BN];
  const T D_f = hll(fl.FD, fr.FD, L.D, R.D);
  const T tau_f = hll(fl.Ftau, fr.Ftau, L.tau, R.tau);
  const T Sn_f = hll(fl.FSn, fr.FSn, X::Sn(L), X::Sn(R));
  const T St1_f = hll(fl.FSt1, fr.FSt1, X::St1(L), X::St1(R));
  const T St2_f = hll(fl.FSt2, fr.FSt2, X::St2(L), X::St2(R));
  // star E, B = HLL averages; cross product E x B by role (:3144-3160)
  const T ErotB_n = Bt2_hll * Et1_hll - Bt1_hll * Et2_hll;
  const T ErotB_t1 = Bn_hll * Et2_hll - Bt2_hll * En_hll;
  const T ErotB_t2 = Bt1_hll * En_hll - Bn_hll * Et1_hll;
  const T E2_perp = pw2(Et1_hll) + pw2(Et2_hll);
  const T B2_perp = pw2(Bt1_hll) + pw2(Bt2_hll);
  // isotropic |E*|^2 + |B*|^2 in x,y,z order
  T Exs, Eys, Ezs, Bxs, Bys, Bzs;
  if constexpr (D == 0) { Exs = En_hll; Eys = Et1_hll; Ezs = Et2_hll; Bxs = Bn_hll; Bys = Bt1_hll; Bzs = Bt2_hll; }
  else                  { Eys = En_hll; Ezs = Et1_hll; Exs = Et2_hll; Bys = Bn_hll; Bzs = Bt1_hll; Bxs = Bt2_hll; }
  const T E2B2_str = T(0.5) * ((pw2(Exs) + pw2(Eys) + pw2(Ezs)) + (pw2(Bxs) + pw2(Bys) + pw2(Bzs)));
  // contact speed (:3208-3335)
  const T a_hll = tau_f - ErotB_n;
  const T b_hll = E2_perp + B2_perp - tau_hll - Sn_f;
  const T c_hll = Sn_hll - ErotB_n;
  const T det_hll = pw2(b_hll) - T(4.0) * a_hll * c_hll;
  const T q_root1 = -T(0.5) * (b_hll + fsgn1(b_hll) * fabs(sqrt(det_hll)));
  T rt2 = c_hll / q_root1;
  if (det_hll < T(0.0)) rt2 = c_hll / b_hll;
  T V = hllc_vel(a_hll, -b_hll, c_hll, rt2, st);
  if (fabs(V) <= T(1.0e-9)) V = T(0.0);
  // star states (:3485-3570)
  const T pstr = Sn_f + (pw2(En_hll) + pw2(Bn_hll)) - (tau_f - ErotB_n) * V;
  const T omV = T(1.0) - V, opV = V + T(1.0);
  const T psiR = (psi_hll - V * En_f) / omV, psiL = (psi_hll + V * En_f) / opV;
  const T phiR = (phi_hll - V * Bn_f) / omV, phiL = (phi_hll + V * Bn_f) / opV;
  const T SnR = (Sn_hll - tau_f * V) / omV, SnL = (Sn_hll + tau_f * V) / opV;
  const T St1R = (St1_hll - St1_f - ErotB_t1 * V - En_hll * Et1_hll - Bn_hll * Bt1_hll) / omV;
  const T St1L = (St1_hll + St1_f + ErotB_t1 * V + En_hll * Et1_hll + Bn_hll * Bt1_hll) / opV;
  const T St2R = (St2_hll - St2_f - ErotB_t2 * V - En_hll * Et2_hll - Bn_hll * Bt2_hll) / omV;
  const T St2L = (St2_hll + St2_f + ErotB_t2 * V + En_hll * Et2_hll + Bn_hll * Bt2_hll) / opV;
  const T tauR = (SnR - ErotB_n) / V - pstr + E2B2_str;
  const T tauL = (SnL - ErotB_n) / V - pstr + E2B2_str;
  const T DR = (D_hll - D_f) / omV, DL = (D_hll + D_f) / opV;
  // HLLC flux selection (:3908-4300): s1 < 0 < v* -> left star flux,
  // v* < 0 < s2 -> right star flux, v* == 0 -> HLL flux.  Only psi, phi, D,
  // tau, S receive the star correction; E, B, q keep the HLL fluxes.
  if (V > T(0.0)) {
    A[R_PSI] = psi_f + (omV * (psiR - psiL)) * h;
    A[R_PHI] = phi_f + (omV * (phiR - phiL)) * h;
    A[R_D] = D_f + omV * (DR - DL) * h;
    A[R_TAU] = tau_f + omV * (tauR - tauL) * h;
    A[R_SN] = Sn_f + omV * (SnR - SnL) * h;
    A[R_ST1] = St1_f + omV * (St1R - St1L) * h;
    A[R_ST2] = St2_f + omV * (St2R - St2L) * h;
  } else if (V < T(0.0)) {
    A[R_PSI] = psi_f + (opV * (psiR - psiL)) * h;
    A[R_PHI] = phi_f + (opV * (phiR - phiL)) * h;
    A[R_D] = D_f + opV * (DR - DL) * h;
    A[R_TAU] = tau_f + opV * (tauR - tauL) * h;
    A[R_SN] = Sn_f + opV * (SnR - SnL) * h;
    A[R_ST1] = St1_f + opV * (St1R - St1L) * h;
    A[R_ST2] = St2_f + opV * (St2R - St2L) * h;
  } else if (V == T(0.0)) {
    A[R_D] = D_f; A[R_TAU] = tau_f; A[R_SN] = Sn_f; A[R_ST1] = St1_f; A[R_ST2] = St2_f;
  } else {
    st |= ST_HLLC_VSTAR;
#pragma unroll
    for (int c = 0; c < NROLE; ++c) A[c] = T(NAN);
  }
}

}  // namespace cueva
