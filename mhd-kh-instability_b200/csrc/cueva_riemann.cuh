// cueva_riemann.cuh -- per-interface HLL / HLLC fluxes of the resistive RMHD
// system, one direction at a time.
//
// Reference: 16_hll_flow_mpx.f95:1358-1965 (HLL),
// 16_hllc_flow_mpx.f95:2401-4618 (HLLC) and 16_hlle_flow_mpx.f95:2526-4614
// (HLLE).  The Fortran writes the x and y
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
static_assert(R_PSI == 0 && R_ET2 == 7, "flux_slot keeps roles 0..7 (psi, phi, E, B) in FP64 for the mixed MP solvers");
static_assert(R_SN == ROLE_SN, "flux_slot keeps the normal momentum flux in FP64 for the split-pressure solvers");

template <typename T>
struct Side {
  T psi, phi, Ex, Ey, Ez, Bx, By, Bz, q, D, tau, Sx, Sy, Sz, vx, vy, vz, p, rho, J;
  T dp;   // split-pressure solvers only: p minus the FP64 reference pressure of the face
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

// physical fluxes of one reconstructed side, 16_hll_flow_mpx.f95:1464-1733;
// h is the enthalpy density rho (1 + eps) + p
template <typename T> struct Phys { T FD, Ftau, FSn, FSt1, FSt2, h; };

// Lorentz factor of the HLL / HLLC routines, 1 / sqrt(1 - (vx^2 + vy^2 + vz^2))
template <typename T>
__device__ __forceinline__ T lorentz(const Side<T>& s) {
  const T V2 = pw2(s.vx) + pw2(s.vy) + pw2(s.vz);
  return T(1.0) / sqrt(T(1.0) - V2);
}
// the HLLE routine subtracts the squares one at a time,
// 1 / sqrt(1 - vx^2 - vy^2 - vz^2) (16_hlle_flow_mpx.f95:2289-2292)
template <typename T>
__device__ __forceinline__ T lorentz_hlle(const Side<T>& s) {
  return T(1.0) / sqrt(T(1.0) - pw2(s.vx) - pw2(s.vy) - pw2(s.vz));
}

// PS (split pressure, mixed precision): the isotropic pressure term of the
// normal momentum flux is s.dp, the side's pressure minus a reference value
// pc0 that the caller adds back in FP64 (the pressure, ~1 in the KH layer,
// would otherwise be rounded to FP32 in a flux whose differences drive the
// small normal velocity)
template <int D, bool PS = false, typename T>
__device__ __forceinline__ Phys<T> physical(const Side<T>& s, T gamma, T W) {
  using X = Dir<D>;
  Phys<T> f;
  const T E2B2 = pw2(s.Ex) + pw2(s.Ey) + pw2(s.Ez) + pw2(s.Bx) + pw2(s.By) + pw2(s.Bz);
  const T eps = s.p / ((gamma - T(1.0)) * s.rho);
  const T h = s.rho * (T(1.0) + eps) + s.p;
  const T hW2 = h * pw2(W);
  const T vn = X::vn(s), vt1 = X::vt1(s), vt2 = X::vt2(s);
  const T En = X::En(s), Et1 = X::Et1(s), Et2 = X::Et2(s);
  const T Bn = X::Bn(s), Bt1 = X::Bt1(s), Bt2 = X::Bt2(s);
  f.FD = s.D * vn;
  f.Ftau = (Bt2 * Et1 - Bt1 * Et2) + hW2 * vn;
  if constexpr (PS) f.FSn = -pw2(En) - pw2(Bn) + hW2 * pw2(vn) + T(0.5) * E2B2 + s.dp;
  else f.FSn = -pw2(En) - pw2(Bn) + hW2 * pw2(vn) + T(0.5) * E2B2 + s.p;
  f.FSt1 = -En * Et1 - Bn * Bt1 + hW2 * vn * vt1;
  if constexpr (D == 0) f.FSt2 = -En * Et2 - Bn * Bt2 + hW2 * vn * vt2;
  else                  f.FSt2 = -En * Et2 - Bn * Bt2 + hW2 * vt2 * vn;   // FSyx: vx before vy
  f.h = h;
  return f;
}
template <int D, bool PS = false, typename T>
__device__ __forceinline__ Phys<T> physical(const Side<T>& s, T gamma) {
  return physical<D, PS>(s, gamma, lorentz(s));
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

// PS: split pressure (see physical); A[R_SN] then lacks the reference
// pressure, which the caller adds in FP64
template <int D, bool PS = false, typename T>
__device__ __forceinline__ void hll_fluxes(const Side<T>& L, const Side<T>& R, T gamma, T* A) {
  using X = Dir<D>;
  em_fluxes<D>(L, R, A);
  const Phys<T> fl = physical<D, PS>(L, gamma), fr = physical<D, PS>(R, gamma);
  A[R_D] = hll(fl.FD, fr.FD, L.D, R.D);
  A[R_TAU] = hll(fl.Ftau, fr.Ftau, L.tau, R.tau);
  A[R_SN] = hll(fl.FSn, fr.FSn, X::Sn(L), X::Sn(R));
  A[R_ST1] = hll(fl.FSt1, fr.FSt1, X::St1(L), X::St1(R));
  A[R_ST2] = hll(fl.FSt2, fr.FSt2, X::St2(L), X::St2(R));
}

// HLL of the second-order MCL routine, 16_hll_flow_mcl.f95:1014-1396 (Sp = 1):
// the fluxes of the MPX HLL with W = 1 / sqrt(1 - vx^2 - vy^2 - vz^2), the
// normal current computed from each side's reconstructed state,
//   J_n = sigma W (E_n + (B_t2 v_t1 - B_t1 v_t2) - (E.v) v_n) + q v_n,
// and the "_m" values of E_t2 and B_t1 (-u + slope, which is not the
// negated side value) in the roles R_BT1 and R_ET2
template <int D, typename T>
__device__ __forceinline__ void mcl_fluxes(const Side<T>& L, const Side<T>& R, const T (&m_et2)[2],
                                           const T (&m_bt1)[2], T gamma, T sigma, T* A) {
  using X = Dir<D>;
  A[R_PSI] = hll(X::En(L), X::En(R), L.psi, R.psi);
  A[R_PHI] = hll(X::Bn(L), X::Bn(R), L.phi, R.phi);
  A[R_BN] = hll(L.phi, R.phi, X::Bn(L), X::Bn(R));
  A[R_BT1] = -hll(m_et2[0], m_et2[1], X::Bt1(L), X::Bt1(R));
  A[R_BT2] = hll(X::Et1(L), X::Et1(R), X::Bt2(L), X::Bt2(R));
  A[R_EN] = hll(L.psi, R.psi, X::En(L), X::En(R));
  A[R_ET1] = hll(X::Bt2(L), X::Bt2(R), X::Et1(L), X::Et1(R));
  A[R_ET2] = -hll(m_bt1[0], m_bt1[1], X::Et2(L), X::Et2(R));
  const T WL = lorentz_hlle(L), WR = lorentz_hlle(R);
  auto jn = [&](const Side<T>& s, T W) {
    const T vrotB = X::Bt2(s) * X::vt1(s) - X::Bt1(s) * X::vt2(s);
    const T Edotv = s.Ex * s.vx + s.Ey * s.vy + s.Ez * s.vz;
    return sigma * W * (X::En(s) + vrotB - Edotv * X::vn(s)) + s.q * X::vn(s);
  };
  A[R_Q] = hll(jn(L, WL), jn(R, WR), L.q, R.q);
  const Phys<T> fl = physical<D>(L, gamma, WL), fr = physical<D>(R, gamma, WR);
  A[R_D] = hll(fl.FD, fr.FD, L.D, R.D);
  A[R_TAU] = hll(fl.Ftau, fr.Ftau, L.tau, R.tau);
  A[R_SN] = hll(fl.FSn, fr.FSn, X::Sn(L), X::Sn(R));
  A[R_ST1] = hll(fl.FSt1, fr.FSt1, X::St1(L), X::St1(R));
  A[R_ST2] = hll(fl.FSt2, fr.FSt2, X::St2(L), X::St2(R));
}

// Lax-Friedrichs cell pairs, 15_lax_flow.f95:749-918 (Sp = 1, const_sp = 0):
// role r transports U with the cell flux F; the face combines p = F + U and
// m = F - U of the cells around it.  The fluid fluxes are flowinit's
// (14_flowinit.f95:258-360): stage E, B, D, S and the time-n v, p and
// hW2 = enthpy W^2, EB = |E|^2 + |B|^2 (each summed x, y, z on its own).
// R_BT1 / R_ET2 carry the reference's sign-flipped cells -E_t2 + B_t1 and
// -B_t1 + E_t2 (EzlaxBy, BylaxEz in x; ExlaxBz, BzlaxEx in y).
template <int D, typename T>
__device__ __forceinline__ void lax_pair(int r, const Side<T>& s, T hW2, T EB, T& F, T& U) {
  using X = Dir<D>;
  switch (r) {
    case R_PSI: F = X::En(s); U = s.psi; break;
    case R_PHI: F = X::Bn(s); U = s.phi; break;
    case R_BN: F = s.phi; U = X::Bn(s); break;
    case R_BT1: F = -X::Et2(s); U = X::Bt1(s); break;
    case R_BT2: F = X::Et1(s); U = X::Bt2(s); break;
    case R_EN: F = s.psi; U = X::En(s); break;
    case R_ET1: F = X::Bt2(s); U = X::Et1(s); break;
    case R_ET2: F = -X::Bt1(s); U = X::Et2(s); break;
    case R_Q: F = s.J; U = s.q; break;
    case R_D: F = s.D * X::vn(s); U = s.D; break;
    case R_TAU: F = (X::Bt2(s) * X::Et1(s) - X::Bt1(s) * X::Et2(s)) + hW2 * X::vn(s); U = s.tau; break;
    case R_SN:
      F = -pw2(X::En(s)) - pw2(X::Bn(s)) + hW2 * pw2(X::vn(s)) + T(0.5) * EB + s.p;
      U = X::Sn(s);
      break;
    case R_ST1: F = -X::En(s) * X::Et1(s) - X::Bn(s) * X::Bt1(s) + hW2 * X::vn(s) * X::vt1(s); U = X::St1(s); break;
    default:   // R_ST2; FSyx multiplies vx before vy
      if constexpr (D == 0) F = -X::En(s) * X::Et2(s) - X::Bn(s) * X::Bt2(s) + hW2 * X::vn(s) * X::vt2(s);
      else                  F = -X::En(s) * X::Et2(s) - X::Bn(s) * X::Bt2(s) + hW2 * X::vt2(s) * X::vn(s);
      U = X::St2(s);
      break;
  }
}
// enthpy W^2 and |E|^2 + |B|^2 of a cell, with startconvar's W and enthalpy
// (06_conserved_var.f95:86-133)
template <typename T>
__device__ __forceinline__ void lax_cell_scalars(const Side<T>& s, T gamma, T& hW2, T& EB) {
  const T W = lorentz(s);
  const T eps = s.p / ((gamma - T(1.0)) * s.rho);
  const T h = s.rho * (T(1.0) + eps) + s.p;
  hW2 = h * pw2(W);
  EB = (pw2(s.Ex) + pw2(s.Ey) + pw2(s.Ez)) + (pw2(s.Bx) + pw2(s.By) + pw2(s.Bz));
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
    if (iter >= 100) {
      if constexpr (sizeof(T) == sizeof(double)) {
        st |= ST_HLLC_NOCONV;
      } else {
        // FP32 (mixed precision): where the quadratic is flat near its root
        // the FP32 steps can hover above the tolerance; the same Newton in
        // FP64 from the same seed decides
        uint32_t st64 = 0;
        v = float(hllc_vel<double>(double(a), double(b), double(c), double(rt), st64));
        st |= st64;
        return v;
      }
      break;
    }
    if (!(err > tol)) break;
  }
  return fmax2(T(-1.0) + T(1.0e-3), fmin2(T(1.0) - T(1.0e-3), v));
}

// HLLC of Miranda-Aranguren et al. (2018), 16_hllc_flow_mpx.f95:2816-4610.
// PS: split pressure with reference pressure pc0 (see physical): the normal
// momentum fluxes and the star pressure lack pc0, which cancels in every
// star-state difference; the contact-speed quadratic takes the full flux.
// A[R_SN] then lacks pc0, which the caller adds in FP64.
template <int D, bool PS = false, typename T>
__device__ __forceinline__ void hllc_fluxes(const Side<T>& L, const Side<T>& R, T gamma, T* A, uint32_t& st,
                                            T* vstar = nullptr, T pc0 = T(0)) {
  using X = Dir<D>;
  em_fluxes<D>(L, R, A);
  const Phys<T> fl = physical<D, PS>(L, gamma), fr = physical<D, PS>(R, gamma);
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
  T b_hll;
  if constexpr (PS) b_hll = E2_perp + B2_perp - tau_hll - (Sn_f + pc0);
  else b_hll = E2_perp + B2_perp - tau_hll - Sn_f;
  const T c_hll = Sn_hll - ErotB_n;
  const T det_hll = pw2(b_hll) - T(4.0) * a_hll * c_hll;
  const T q_root1 = -T(0.5) * (b_hll + fsgn1(b_hll) * fabs(sqrt(det_hll)));
  T rt2 = c_hll / q_root1;
  if (det_hll < T(0.0)) rt2 = c_hll / b_hll;
  T V = hllc_vel(a_hll, -b_hll, c_hll, rt2, st);
  if (fabs(V) <= T(1.0e-9)) V = T(0.0);
  if (vstar) *vstar = V;   // the contact speed the flux choice below uses
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

// HLLE variant, 16_hlle_flow_mpx.f95 (2D, :2526-4614).  psi, phi, E and B
// keep the fixed-speed HLL fluxes (their star fluxes are the HLL ones,
// :3489-3604; the flux choice :3881-4019 takes them in both branches); q, D,
// tau and S use the bounds s1 = min(lambda-), s2 = max(lambda+) of the
// relativistic sound speed (:2709-2826, the reference writes vn where the
// textbook bound has vn^2 under the root), and D, tau, S receive the
// HLLC-type contact of the same quadratic for v* (:3165-3420).  Flux choice
// (:4021-4286): s1 >= 0 left physical flux, s1 <= 0 <= v* left star flux,
// v* <= 0 <= s2 right star flux, s2 < 0 right physical flux.  No superluminal
// or density fix-ups precede this solver.
template <int D, typename T>
__device__ __forceinline__ void hlle_bounds(const Side<T>& s, T h, T gamma, T& lm, T& lp) {
  using X = Dir<D>;
  const T vn = X::vn(s);
  const T Cs = sqrt(gamma * s.p / (h));
  const T V2 = pw2(s.vx) + pw2(s.vy) + pw2(s.vz);
  const T root = sqrt((T(1.0) - V2) * (T(1.0) - V2 * pw2(Cs) - vn * (T(1.0) - pw2(Cs))));
  lp = (vn * (T(1.0) - pw2(Cs)) + Cs * root) / (T(1.0) - pw2(Cs) * V2);
  lm = (vn * (T(1.0) - pw2(Cs)) - Cs * root) / (T(1.0) - pw2(Cs) * V2);
}

// PS: split pressure with reference pressure pc0, as in hllc_fluxes
template <int D, bool PS = false, typename T>
__device__ __forceinline__ void hlle_fluxes(const Side<T>& L, const Side<T>& R, T gamma, T* A, uint32_t& st,
                                            T pc0 = T(0)) {
  using X = Dir<D>;
  em_fluxes<D>(L, R, A);   // psi, phi, E, B; the charge flux is replaced below
  const Phys<T> fl = physical<D, PS>(L, gamma, lorentz_hlle(L)), fr = physical<D, PS>(R, gamma, lorentz_hlle(R));
  const T h = T(0.5);
  // fixed-speed HLL states of E and B (the star E, B)
  const T En_hll = h * (((X::En(R) + X::En(L)) + L.psi) - R.psi);
  const T Et1_hll = h * (((X::Et1(R) + X::Et1(L)) + X::Bt2(L)) - X::Bt2(R));
  const T Et2_hll = h * (((X::Et2(R) + X::Et2(L)) - X::Bt1(L)) + X::Bt1(R));
  const T Bn_hll = h * (((X::Bn(R) + X::Bn(L)) + L.phi) - R.phi);
  const T Bt1_hll = h * (((X::Bt1(R) + X::Bt1(L)) - X::Et2(L)) + X::Et2(R));
  const T Bt2_hll = h * (((X::Bt2(R) + X::Bt2(L)) + X::Et1(L)) - X::Et1(R));
  // wave bounds (:2796-2819: NaN stops the reference; |s| > 1 is clamped)
  T lmL, lpL, lmR, lpR;
  hlle_bounds<D>(R, fr.h, gamma, lmR, lpR);
  hlle_bounds<D>(L, fl.h, gamma, lmL, lpL);
  T s1 = fmin2(lmL, lmR), s2 = fmax2(lpL, lpR);
  if (isnan(s1) || isnan(s2)) st |= ST_HLLE_SPEED;
  const T eps2 = T(1.0e-9);
  if (fabs(s1) > T(1.0)) s1 = fmax2(T(-1.0) + eps2, fmin2(T(1.0) - eps2, s1));
  if (fabs(s2) > T(1.0)) s2 = fmax2(T(-1.0) + eps2, fmin2(T(1.0) - eps2, s2));
  // fluid HLL states and HLLE fluxes with the bounds
  const T D_hll = (s2 * R.D - s1 * L.D + fl.FD - fr.FD) / (s2 - s1);
  const T tau_hll = (s2 * R.tau - s1 * L.tau + fl.Ftau - fr.Ftau) / (s2 - s1);
  const T Sn_hll = (s2 * X::Sn(R) - s1 * X::Sn(L) + fl.FSn - fr.FSn) / (s2 - s1);
  const T St1_hll = (s2 * X::St1(R) - s1 * X::St1(L) + fl.FSt1 - fr.FSt1) / (s2 - s1);
  const T St2_hll = (s2 * X::St2(R) - s1 * X::St2(L) + fl.FSt2 - fr.FSt2) / (s2 - s1);
  auto hlle = [&](T FL, T FR, T UL, T UR) { return (s2 * FL - s1 * FR + s1 * s2 * (UR - UL)) / (s2 - s1); };
  const T q_f = hlle(L.J, R.J, L.q, R.q);
  const T D_f = hlle(fl.FD, fr.FD, L.D, R.D);
  const T tau_f = hlle(fl.Ftau, fr.Ftau, L.tau, R.tau);
  const T Sn_f = hlle(fl.FSn, fr.FSn, X::Sn(L), X::Sn(R));
  const T St1_f = hlle(fl.FSt1, fr.FSt1, X::St1(L), X::St1(R));
  const T St2_f = hlle(fl.FSt2, fr.FSt2, X::St2(L), X::St2(R));
  // contact speed of the HLLC quadratic, with the HLLE states and fluxes
  const T ErotB_n = Bt2_hll * Et1_hll - Bt1_hll * Et2_hll;
  const T ErotB_t1 = Bn_hll * Et2_hll - Bt2_hll * En_hll;
  const T ErotB_t2 = Bt1_hll * En_hll - Bn_hll * Et1_hll;
  const T E2_perp = pw2(Et1_hll) + pw2(Et2_hll);
  const T B2_perp = pw2(Bt1_hll) + pw2(Bt2_hll);
  T Exs, Eys, Ezs, Bxs, Bys, Bzs;
  if constexpr (D == 0) { Exs = En_hll; Eys = Et1_hll; Ezs = Et2_hll; Bxs = Bn_hll; Bys = Bt1_hll; Bzs = Bt2_hll; }
  else                  { Eys = En_hll; Ezs = Et1_hll; Exs = Et2_hll; Bys = Bn_hll; Bzs = Bt1_hll; Bxs = Bt2_hll; }
  const T E2B2_str = T(0.5) * ((pw2(Exs) + pw2(Eys) + pw2(Ezs)) + (pw2(Bxs) + pw2(Bys) + pw2(Bzs)));
  const T a_hll = tau_f - ErotB_n;
  T b_hll;
  if constexpr (PS) b_hll = E2_perp + B2_perp - tau_hll - (Sn_f + pc0);
  else b_hll = E2_perp + B2_perp - tau_hll - Sn_f;
  const T c_hll = Sn_hll - ErotB_n;
  const T det_hll = pw2(b_hll) - T(4.0) * a_hll * c_hll;
  const T q_root1 = -T(0.5) * (b_hll + fsgn1(b_hll) * fabs(sqrt(det_hll)));
  T rt2 = c_hll / q_root1;
  if (det_hll < T(0.0)) rt2 = c_hll / b_hll;
  T V = hllc_vel(a_hll, -b_hll, c_hll, rt2, st);
  if (fabs(V) <= T(1.0e-9)) V = T(0.0);
  // star states (:3378-3420)
  const T pstr = Sn_f + (pw2(En_hll) + pw2(Bn_hll)) - (tau_f - ErotB_n) * V;
  const T SnR = (s2 * Sn_hll - tau_f * V) / (s2 - V);
  const T SnL = (-s1 * Sn_hll + tau_f * V) / (V - s1);
  const T St1R = (s2 * St1_hll - St1_f - ErotB_t1 * V - En_hll * Et1_hll - Bn_hll * Bt1_hll) / (s2 - V);
  const T St1L = (-s1 * St1_hll + St1_f + ErotB_t1 * V + En_hll * Et1_hll + Bn_hll * Bt1_hll) / (V - s1);
  const T St2R = (s2 * St2_hll - St2_f - ErotB_t2 * V - En_hll * Et2_hll - Bn_hll * Bt2_hll) / (s2 - V);
  const T St2L = (-s1 * St2_hll + St2_f + ErotB_t2 * V + En_hll * Et2_hll + Bn_hll * Bt2_hll) / (V - s1);
  const T tauR = (SnR - ErotB_n) / V - pstr + E2B2_str;
  const T tauL = (SnL - ErotB_n) / V - pstr + E2B2_str;
  const T DR = (s2 * D_hll - D_f) / (s2 - V);
  const T DL = (-s1 * D_hll + D_f) / (V - s1);
  // star fluxes (:3489-3604; v* == 0 keeps the HLLE fluxes)
  T fDR = D_f, fDL = D_f, ftR = tau_f, ftL = tau_f, fSnR = Sn_f, fSnL = Sn_f, fS1R = St1_f, fS1L = St1_f,
    fS2R = St2_f, fS2L = St2_f;
  if (V != T(0.0)) {
    fDR = D_f + s2 * (V - s1) * (DR - DL) / (s2 - s1);
    fDL = D_f - s1 * (s2 - V) * (DR - DL) / (s2 - s1);
    ftR = tau_f + s2 * (V - s1) * (tauR - tauL) / (s2 - s1);
    ftL = tau_f - s1 * (s2 - V) * (tauR - tauL) / (s2 - s1);
    fSnR = Sn_f + s2 * (V - s1) * (SnR - SnL) / (s2 - s1);
    fSnL = Sn_f - s1 * (s2 - V) * (SnR - SnL) / (s2 - s1);
    fS1R = St1_f + s2 * (V - s1) * (St1R - St1L) / (s2 - s1);
    fS1L = St1_f - s1 * (s2 - V) * (St1R - St1L) / (s2 - s1);
    fS2R = St2_f + s2 * (V - s1) * (St2R - St2L) / (s2 - s1);
    fS2L = St2_f - s1 * (s2 - V) * (St2R - St2L) / (s2 - s1);
  }
  if (s1 >= T(0.0)) {
    A[R_Q] = L.J; A[R_D] = fl.FD; A[R_TAU] = fl.Ftau; A[R_SN] = fl.FSn; A[R_ST1] = fl.FSt1; A[R_ST2] = fl.FSt2;
  } else if (s1 <= T(0.0) && T(0.0) <= V) {
    A[R_Q] = q_f; A[R_D] = fDL; A[R_TAU] = ftL; A[R_SN] = fSnL; A[R_ST1] = fS1L; A[R_ST2] = fS2L;
  } else if (V <= T(0.0) && T(0.0) <= s2) {
    A[R_Q] = q_f; A[R_D] = fDR; A[R_TAU] = ftR; A[R_SN] = fSnR; A[R_ST1] = fS1R; A[R_ST2] = fS2R;
  } else if (s2 < T(0.0)) {
    A[R_Q] = R.J; A[R_D] = fr.FD; A[R_TAU] = fr.Ftau; A[R_SN] = fr.FSn; A[R_ST1] = fr.FSt1; A[R_ST2] = fr.FSt2;
  } else {   // the reference stops (:4284-4285, 4612-4613)
    st |= ST_HLLC_VSTAR;
    A[R_Q] = A[R_D] = A[R_TAU] = A[R_SN] = A[R_ST1] = A[R_ST2] = T(NAN);
  }
}

// HLLC of the MC family, 16_hllc_flow_mcl.f95 (2D :1751-4056): the HLLC of
// hllc_fluxes (same HLL states, star states and flux choice, s = -1, +1) on
// the MC sides -- the "_m" values of E_t2 and B_t1 in the HLL states and
// fluxes, the current of each side, W = 1 / sqrt(1 - vx^2 - vy^2 - vz^2) --
// with |v*| <= 1e-6 taken as 0 (:2580-2600; the MPX routine uses 1e-9).
template <int D, typename T>
__device__ __forceinline__ void hllcmc_fluxes(const Side<T>& L, const Side<T>& R, const T (&m_et2)[2],
                                              const T (&m_bt1)[2], T gamma, T sigma, T* A, uint32_t& st,
                                              T* vstar = nullptr) {
  using X = Dir<D>;
  mcl_fluxes<D>(L, R, m_et2, m_bt1, gamma, sigma, A);   // fixed-speed HLL fluxes of every role
  const Phys<T> fl = physical<D>(L, gamma, lorentz_hlle(L)), fr = physical<D>(R, gamma, lorentz_hlle(R));
  const T h = T(0.5);
  const T psi_hll = h * (((R.psi + L.psi) + X::En(L)) - X::En(R));
  const T phi_hll = h * (((R.phi + L.phi) + X::Bn(L)) - X::Bn(R));
  const T En_hll = h * (((X::En(R) + X::En(L)) + L.psi) - R.psi);
  const T Et1_hll = h * (((X::Et1(R) + X::Et1(L)) + X::Bt2(L)) - X::Bt2(R));
  const T Et2_hll = h * (((X::Et2(R) + X::Et2(L)) + m_bt1[0]) - m_bt1[1]);
  const T Bn_hll = h * (((X::Bn(R) + X::Bn(L)) + L.phi) - R.phi);
  const T Bt1_hll = h * (((X::Bt1(R) + X::Bt1(L)) + m_et2[0]) - m_et2[1]);
  const T Bt2_hll = h * (((X::Bt2(R) + X::Bt2(L)) + X::Et1(L)) - X::Et1(R));
  const T D_hll = h * (((R.D + L.D) + fl.FD) - fr.FD);
  const T tau_hll = h * (((R.tau + L.tau) + fl.Ftau) - fr.Ftau);
  const T Sn_hll = h * (((X::Sn(R) + X::Sn(L)) + fl.FSn) - fr.FSn);
  const T St1_hll = h * (((X::St1(R) + X::St1(L)) + fl.FSt1) - fr.FSt1);
  const T St2_hll = h * (((X::St2(R) + X::St2(L)) + fl.FSt2) - fr.FSt2);
  const T psi_f = A[R_PSI], phi_f = A[R_PHI], En_f = A[R_EN], Bn_f = A[R_BN];
  const T D_f = A[R_D], tau_f = A[R_TAU], Sn_f = A[R_SN], St1_f = A[R_ST1], St2_f = A[R_ST2];
  const T ErotB_n = Bt2_hll * Et1_hll - Bt1_hll * Et2_hll;
  const T ErotB_t1 = Bn_hll * Et2_hll - Bt2_hll * En_hll;
  const T ErotB_t2 = Bt1_hll * En_hll - Bn_hll * Et1_hll;
  const T E2_perp = pw2(Et1_hll) + pw2(Et2_hll);
  const T B2_perp = pw2(Bt1_hll) + pw2(Bt2_hll);
  T Exs, Eys, Ezs, Bxs, Bys, Bzs;
  if constexpr (D == 0) { Exs = En_hll; Eys = Et1_hll; Ezs = Et2_hll; Bxs = Bn_hll; Bys = Bt1_hll; Bzs = Bt2_hll; }
  else                  { Eys = En_hll; Ezs = Et1_hll; Exs = Et2_hll; Bys = Bn_hll; Bzs = Bt1_hll; Bxs = Bt2_hll; }
  const T E2B2_str = T(0.5) * ((pw2(Exs) + pw2(Eys) + pw2(Ezs)) + (pw2(Bxs) + pw2(Bys) + pw2(Bzs)));
  const T a_hll = tau_f - ErotB_n;
  const T b_hll = E2_perp + B2_perp - tau_hll - Sn_f;
  const T c_hll = Sn_hll - ErotB_n;
  const T det_hll = pw2(b_hll) - T(4.0) * a_hll * c_hll;
  const T q_root1 = -T(0.5) * (b_hll + fsgn1(b_hll) * fabs(sqrt(det_hll)));
  T rt2 = c_hll / q_root1;
  if (det_hll < T(0.0)) rt2 = c_hll / b_hll;
  T V = hllc_vel(a_hll, -b_hll, c_hll, rt2, st);
  if (fabs(V) <= T(1.0e-6)) V = T(0.0);
  if (vstar) *vstar = V;   // the contact speed the flux choice below uses
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
  // flux choice (:3530-3620): v* > 0 left star flux, v* < 0 right star flux,
  // v* == 0 the HLL fluxes; E, B and q keep the HLL fluxes throughout
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
  } else if (!(V == T(0.0))) {
    st |= ST_HLLC_VSTAR;
#pragma unroll
    for (int c = 0; c < NROLE; ++c) A[c] = T(NAN);
  }
}

// HLLE of the MC family, 16_hlle_flow_mcl.f95 (2D :1638-4345), on the MC
// reconstruction with the "_m" values of E_t2 and B_t1 and the current
// of each side (as mcl_fluxes).  Bounds and the v* quadratic are the
// MPX HLLE's; the star states and fluxes differ (:2911-3150):
//   S_n*  = (s S_n,hll - F(S_n)_hll +- (p* - B_n*^2 - E_n*^2 - (E*xB*)_n v*)) / (s - v*)
//   tau*  = (s tau_hll - F(tau)_hll +- ((p* - |E*|^2/2 - |B*|^2/2) v* + (E*xB*)_n)) / (s - v*)
//   F*    = F(side) + s (U* - U(side)),   s = s1 (left) or s2 (right);
// the EM fluxes for v* != 0 are those of the star state (psi: E_n*,
// E_n: psi*, E_t1: B_t2*, E_t2: -B_t1*, B_n: phi*, B_t1: -E_t2*,
// B_t2: E_t1*), for v* == 0 the fixed-speed HLL ones; the current flux is
// the HLLE one in both star regions.  Flux choice (:3236-4343): s1 > 0
// left physical flux, s1 <= 0 <= v* left star, v* < 0 <= s2 right star,
// s2 < 0 right physical flux.  A NaN v* leaves the reference's EM arrays
// unset (and its fluid choice stops the run); both are reported as
// ST_HLLC_VSTAR with NaN fluxes here.
template <int D, typename T>
__device__ __forceinline__ void hllemc_fluxes(const Side<T>& L, const Side<T>& R, const T (&m_et2)[2],
                                              const T (&m_bt1)[2], T gamma, T sigma, T* A, uint32_t& st) {
  using X = Dir<D>;
  const T h = T(0.5);
  // fixed-speed HLL states (the star E, B, psi, phi)
  const T psi_hll = h * (((R.psi + L.psi) + X::En(L)) - X::En(R));
  const T phi_hll = h * (((R.phi + L.phi) + X::Bn(L)) - X::Bn(R));
  const T En_hll = h * (((X::En(R) + X::En(L)) + L.psi) - R.psi);
  const T Et1_hll = h * (((X::Et1(R) + X::Et1(L)) + X::Bt2(L)) - X::Bt2(R));
  const T Et2_hll = h * (((X::Et2(R) + X::Et2(L)) + m_bt1[0]) - m_bt1[1]);
  const T Bn_hll = h * (((X::Bn(R) + X::Bn(L)) + L.phi) - R.phi);
  const T Bt1_hll = h * (((X::Bt1(R) + X::Bt1(L)) + m_et2[0]) - m_et2[1]);
  const T Bt2_hll = h * (((X::Bt2(R) + X::Bt2(L)) + X::Et1(L)) - X::Et1(R));
  const T WL = lorentz_hlle(L), WR = lorentz_hlle(R);
  const Phys<T> fl = physical<D>(L, gamma, WL), fr = physical<D>(R, gamma, WR);
  auto jn = [&](const Side<T>& s, T W) {
    const T vrotB = X::Bt2(s) * X::vt1(s) - X::Bt1(s) * X::vt2(s);
    const T Edotv = s.Ex * s.vx + s.Ey * s.vy + s.Ez * s.vz;
    return sigma * W * (X::En(s) + vrotB - Edotv * X::vn(s)) + s.q * X::vn(s);
  };
  const T JL = jn(L, WL), JR = jn(R, WR);
  T lmL, lpL, lmR, lpR;
  hlle_bounds<D>(R, fr.h, gamma, lmR, lpR);
  hlle_bounds<D>(L, fl.h, gamma, lmL, lpL);
  T s1 = fmin2(lmL, lmR), s2 = fmax2(lpL, lpR);
  if (isnan(s1) || isnan(s2)) st |= ST_HLLE_SPEED;
  const T eps2 = T(1.0e-9);
  if (fabs(s1) > T(1.0)) s1 = fmax2(T(-1.0) + eps2, fmin2(T(1.0) - eps2, s1));
  if (fabs(s2) > T(1.0)) s2 = fmax2(T(-1.0) + eps2, fmin2(T(1.0) - eps2, s2));
  const T D_hll = (s2 * R.D - s1 * L.D + fl.FD - fr.FD) / (s2 - s1);
  const T tau_hll = (s2 * R.tau - s1 * L.tau + fl.Ftau - fr.Ftau) / (s2 - s1);
  const T Sn_hll = (s2 * X::Sn(R) - s1 * X::Sn(L) + fl.FSn - fr.FSn) / (s2 - s1);
  const T St1_hll = (s2 * X::St1(R) - s1 * X::St1(L) + fl.FSt1 - fr.FSt1) / (s2 - s1);
  const T St2_hll = (s2 * X::St2(R) - s1 * X::St2(L) + fl.FSt2 - fr.FSt2) / (s2 - s1);
  auto hlle = [&](T FL, T FR, T UL, T UR) { return (s2 * FL - s1 * FR + s1 * s2 * (UR - UL)) / (s2 - s1); };
  const T q_f = hlle(JL, JR, L.q, R.q);
  const T D_f = hlle(fl.FD, fr.FD, L.D, R.D);
  const T tau_f = hlle(fl.Ftau, fr.Ftau, L.tau, R.tau);
  const T Sn_f = hlle(fl.FSn, fr.FSn, X::Sn(L), X::Sn(R));
  const T St1_f = hlle(fl.FSt1, fr.FSt1, X::St1(L), X::St1(R));
  const T St2_f = hlle(fl.FSt2, fr.FSt2, X::St2(L), X::St2(R));
  const T ErotB_n = Bt2_hll * Et1_hll - Bt1_hll * Et2_hll;
  const T ErotB_t1 = Bn_hll * Et2_hll - Bt2_hll * En_hll;
  const T ErotB_t2 = Bt1_hll * En_hll - Bn_hll * Et1_hll;
  const T E2_perp = pw2(Et1_hll) + pw2(Et2_hll);
  const T B2_perp = pw2(Bt1_hll) + pw2(Bt2_hll);
  T Exs, Eys, Ezs, Bxs, Bys, Bzs;
  if constexpr (D == 0) { Exs = En_hll; Eys = Et1_hll; Ezs = Et2_hll; Bxs = Bn_hll; Bys = Bt1_hll; Bzs = Bt2_hll; }
  else                  { Eys = En_hll; Ezs = Et1_hll; Exs = Et2_hll; Bys = Bn_hll; Bzs = Bt1_hll; Bxs = Bt2_hll; }
  const T E2B2_str = T(0.5) * ((pw2(Exs) + pw2(Eys) + pw2(Ezs)) + (pw2(Bxs) + pw2(Bys) + pw2(Bzs)));
  const T a_hll = tau_f - ErotB_n;
  const T b_hll = E2_perp + B2_perp - tau_hll - Sn_f;
  const T c_hll = Sn_hll - ErotB_n;
  const T det_hll = pw2(b_hll) - T(4.0) * a_hll * c_hll;
  const T q_root1 = -T(0.5) * (b_hll + fsgn1(b_hll) * fabs(sqrt(det_hll)));
  T rt2 = c_hll / q_root1;
  if (det_hll < T(0.0)) rt2 = c_hll / b_hll;
  T V = hllc_vel(a_hll, -b_hll, c_hll, rt2, st);
  if (fabs(V) <= T(1.0e-9)) V = T(0.0);
  // star states
  const T pstr = Sn_f + (pw2(En_hll) + pw2(Bn_hll)) - (tau_f - ErotB_n) * V;
  const T SnR = (s2 * Sn_hll - Sn_f + pstr - pw2(Bn_hll) - pw2(En_hll) - ErotB_n * V) / (s2 - V);
  const T SnL = (-s1 * Sn_hll + Sn_f - pstr + pw2(Bn_hll) + pw2(En_hll) + ErotB_n * V) / (V - s1);
  const T St1R = (s2 * St1_hll - St1_f - ErotB_t1 * V - En_hll * Et1_hll - Bn_hll * Bt1_hll) / (s2 - V);
  const T St1L = (-s1 * St1_hll + St1_f + ErotB_t1 * V + En_hll * Et1_hll + Bn_hll * Bt1_hll) / (V - s1);
  const T St2R = (s2 * St2_hll - St2_f - ErotB_t2 * V - En_hll * Et2_hll - Bn_hll * Bt2_hll) / (s2 - V);
  const T St2L = (-s1 * St2_hll + St2_f + ErotB_t2 * V + En_hll * Et2_hll + Bn_hll * Bt2_hll) / (V - s1);
  const T tauR = (s2 * tau_hll - tau_f + (pstr - E2B2_str) * V + ErotB_n) / (s2 - V);
  const T tauL = (-s1 * tau_hll + tau_f - (pstr - E2B2_str) * V - ErotB_n) / (V - s1);
  const T DR = (s2 * D_hll - D_f) / (s2 - V);
  const T DL = (-s1 * D_hll + D_f) / (V - s1);
  // star fluxes
  T fDR = D_f, fDL = D_f, ftR = tau_f, ftL = tau_f, fSnR = Sn_f, fSnL = Sn_f, fS1R = St1_f, fS1L = St1_f,
    fS2R = St2_f, fS2L = St2_f;
  if (V == T(0.0)) {
    A[R_PSI] = hll(X::En(L), X::En(R), L.psi, R.psi);
    A[R_PHI] = hll(X::Bn(L), X::Bn(R), L.phi, R.phi);
    A[R_BN] = hll(L.phi, R.phi, X::Bn(L), X::Bn(R));
    A[R_BT1] = -hll(m_et2[0], m_et2[1], X::Bt1(L), X::Bt1(R));
    A[R_BT2] = hll(X::Et1(L), X::Et1(R), X::Bt2(L), X::Bt2(R));
    A[R_EN] = hll(L.psi, R.psi, X::En(L), X::En(R));
    A[R_ET1] = hll(X::Bt2(L), X::Bt2(R), X::Et1(L), X::Et1(R));
    A[R_ET2] = -hll(m_bt1[0], m_bt1[1], X::Et2(L), X::Et2(R));
  } else if (V == V) {
    // flux of the star state; R_BT1 / R_ET2 hold -F(B_t1) = E_t2*, -F(E_t2) = B_t1*
    A[R_PSI] = En_hll; A[R_PHI] = Bn_hll; A[R_BN] = phi_hll; A[R_BT1] = Et2_hll;
    A[R_BT2] = Et1_hll; A[R_EN] = psi_hll; A[R_ET1] = Bt2_hll; A[R_ET2] = Bt1_hll;
    fDR = fr.FD + s2 * (DR - R.D);                 fDL = fl.FD + s1 * (DL - L.D);
    ftR = fr.Ftau + s2 * (tauR - R.tau);           ftL = fl.Ftau + s1 * (tauL - L.tau);
    fSnR = fr.FSn + s2 * (SnR - X::Sn(R));         fSnL = fl.FSn + s1 * (SnL - X::Sn(L));
    fS1R = fr.FSt1 + s2 * (St1R - X::St1(R));      fS1L = fl.FSt1 + s1 * (St1L - X::St1(L));
    fS2R = fr.FSt2 + s2 * (St2R - X::St2(R));      fS2L = fl.FSt2 + s1 * (St2L - X::St2(L));
  } else {
    st |= ST_HLLC_VSTAR;
#pragma unroll
    for (int c = R_PSI; c <= R_ET2; ++c) A[c] = T(NAN);
  }
  if (s1 > T(0.0)) {
    A[R_Q] = JL; A[R_D] = fl.FD; A[R_TAU] = fl.Ftau; A[R_SN] = fl.FSn; A[R_ST1] = fl.FSt1; A[R_ST2] = fl.FSt2;
  } else if (s1 <= T(0.0) && T(0.0) <= V) {
    A[R_Q] = q_f; A[R_D] = fDL; A[R_TAU] = ftL; A[R_SN] = fSnL; A[R_ST1] = fS1L; A[R_ST2] = fS2L;
  } else if (V < T(0.0) && T(0.0) <= s2) {
    A[R_Q] = q_f; A[R_D] = fDR; A[R_TAU] = ftR; A[R_SN] = fSnR; A[R_ST1] = fS1R; A[R_ST2] = fS2R;
  } else if (s2 < T(0.0)) {
    A[R_Q] = JR; A[R_D] = fr.FD; A[R_TAU] = fr.Ftau; A[R_SN] = fr.FSn; A[R_ST1] = fr.FSt1; A[R_ST2] = fr.FSt2;
  } else {   // the reference stops
    st |= ST_HLLC_VSTAR;
    A[R_Q] = A[R_D] = A[R_TAU] = A[R_SN] = A[R_ST1] = A[R_ST2] = T(NAN);
  }
}

}  // namespace cueva
