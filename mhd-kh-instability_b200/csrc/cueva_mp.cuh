// cueva_mp.cuh -- MP5 / MP7 / MP9 monotonicity-preserving reconstruction
// (Suresh & Huynh 1997) as one interface pair per thread.
//
// The reference reconstructs whole grid lines (mp5.f95:2-278, mp7.f95:2-315,
// mp9.f95:2-320): for every cell k it forms the limited left value up(k) at
// k+1/2 and right value um(k) at k-1/2, and the interface between cells i and
// i+1 takes L = up(i), R = um(i+1) (16_hll_flow_mpx.f95:942-1036).  Every
// (cell, slot) value depends only on the cells k-R..k+R of its own slot, so a
// thread that owns interface i loads the 2R+2 cells i-R..i+1+R into registers
// and evaluates exactly the two values it needs.  Operation order follows the
// Fortran so the FP64 build without FMA contraction is bit-identical.
#pragma once
#include "cueva_common.cuh"

namespace cueva {

// The minmod functions of funciones.f95 are written with sign arithmetic,
//   DMM(x, y)      = 0.5 (sign(1,x) + sign(1,y)) min(|x|, |y|)          (:148-162)
//   DM4(w, x, y, z) = 0.125 (sign(1,w) + sign(1,x))
//                     |(sign(1,w) + sign(1,y)) (sign(1,w) + sign(1,z))| min(|w|,|x|,|y|,|z|)   (:165-185)
// Every factor in front of the minimum is exactly +-1 or a signed zero, so
// they equal a selection on the sign bits: +-min with the sign of the first
// argument where all signs agree; otherwise (+-0) * min, with -0 only where
// DM4's first pair agrees (0.125 (+-2) |0| = -0 for negative w).  The zero
// is still multiplied by the minimum so that an infinite or NaN minimum
// gives NaN as in the sign arithmetic.  Results are bit-identical, with a
// third of the FP64 operations (the MP limiters call these in every pair).
template <typename T>
__device__ __forceinline__ T DMM(T x, T y) {
  const T m = fmin2(fabs(x), fabs(y));
  return (signbit(x) == signbit(y)) ? copysign(m, x) : T(0) * m;
}
template <typename T>
__device__ __forceinline__ T DM4(T w, T xx, T y, T z) {
  const T m = fmin2(fmin2(fmin2(fabs(w), fabs(xx)), fabs(y)), fabs(z));
  const bool sw = signbit(w);
  const bool first = signbit(xx) == sw;
  if (first && signbit(y) == sw && signbit(z) == sw) return copysign(m, w);
  return (first ? copysign(T(0), w) : T(0)) * m;
}

// stencil radius of the unlimited interface formula; RM = 3 is the
// second-order MC reconstruction of the MCL flux routines (radius 1)
template <int RM> struct MPR { static constexpr int R = RM + 2; };
template <> struct MPR<3> { static constexpr int R = 1; };

// monotonized-central slope (mcl with slop = 2, funciones.f95:56-95):
// 0.5 (sign(1,a) + sign(1,b)) min(2|a|, 2|b|, |a+b|/2), the sign factor
// taken as a selection on the sign bits as in DMM
template <typename T>
__device__ __forceinline__ T mc_slope(T fa, T fb) {
  const T m = fmin2(fmin2(T(2.0) * fabs(fa), T(2.0) * fabs(fb)), T(0.5) * fabs(fa + fb));
  return (signbit(fa) == signbit(fb)) ? copysign(m, fa) : T(0) * m;
}

// unlimited left value at k+1/2 (SH97 eq. 2.1 / 2.31) around register index C
template <int RM, int C, typename T, int N>
__device__ __forceinline__ T mp_vorp(const T (&u)[N]) {
  if constexpr (RM == 0) {
    const T b1 = T(1.0 / 60.0);
    return b1 * (T(2.0) * u[C - 2] - T(13.0) * u[C - 1] + T(47.0) * u[C] + T(27.0) * u[C + 1] - T(3.0) * u[C + 2]);
  } else if constexpr (RM == 1) {
    const T b1 = T(1.0 / 420.0);
    return b1 * (-T(3.0) * u[C - 3] + T(25.0) * u[C - 2] - T(101.0) * u[C - 1] + T(319.0) * u[C] +
                 T(214.0) * u[C + 1] - T(38.0) * u[C + 2] + T(4.0) * u[C + 3]);
  } else {
    const T b1 = T(1.0 / 2520.0);
    return b1 * (T(4.0) * u[C - 4] - T(41.0) * u[C - 3] + T(199.0) * u[C - 2] - T(641.0) * u[C - 1] +
                 T(1879.0) * u[C] + T(1375.0) * u[C + 1] - T(305.0) * u[C + 2] + T(55.0) * u[C + 3] -
                 T(5.0) * u[C + 4]);
  }
}
// unlimited right value at k-1/2 (mirror formulas, same term order as the Fortran)
template <int RM, int C, typename T, int N>
__device__ __forceinline__ T mp_vorm(const T (&u)[N]) {
  if constexpr (RM == 0) {
    const T b1 = T(1.0 / 60.0);
    return b1 * (-T(3.0) * u[C - 2] + T(27.0) * u[C - 1] + T(47.0) * u[C] - T(13.0) * u[C + 1] + T(2.0) * u[C + 2]);
  } else if constexpr (RM == 1) {
    const T b1 = T(1.0 / 420.0);
    return b1 * (-T(3.0) * u[C + 3] + T(25.0) * u[C + 2] - T(101.0) * u[C + 1] + T(319.0) * u[C] +
                 T(214.0) * u[C - 1] - T(38.0) * u[C - 2] + T(4.0) * u[C - 3]);
  } else {
    const T b1 = T(1.0 / 2520.0);
    return b1 * (T(4.0) * u[C + 4] - T(41.0) * u[C + 3] + T(199.0) * u[C + 2] - T(641.0) * u[C + 1] +
                 T(1879.0) * u[C] + T(1375.0) * u[C - 1] - T(305.0) * u[C - 2] + T(55.0) * u[C - 3] -
                 T(5.0) * u[C - 4]);
  }
}

// up(k) for the cell at register index C (mp5.f95:104-136) in two steps:
// mp_up_fast gives the unlimited value vorp and whether it passes the
// monotonicity test (then vorp is up(k)); mp_up_lim gives the limited value
// of a vorp that failed it.  mp_up chains them; the interface pairs below
// take all their tests first (independent chains for the scheduler) and
// limit only the values that failed.  The operations are the same.
template <int RM, int C, typename T, int N>
__device__ __forceinline__ T mp_up_fast(const T (&u)[N], bool& ok) {
  const T alpha = T(2.0), epsm = T(1.0e-10);
  const T du0 = u[C] - u[C - 1];
  const T du1 = u[C + 1] - u[C];
  const T vorp = mp_vorp<RM, C>(u);
  const T vmpp = u[C] + DMM(du1, alpha * du0);
  ok = (vorp - u[C]) * (vorp - vmpp) <= epsm;
  return vorp;
}
template <int RM, int C, typename T, int N>
__device__ __forceinline__ T mp_up_lim(const T (&u)[N], T vorp) {
  const T alpha = T(2.0), b2 = T(4.0 / 3.0);
  const T du0 = u[C] - u[C - 1];
  const T d2m = u[C - 2] - T(2.0) * u[C - 1] + u[C];
  const T d20 = u[C - 1] - T(2.0) * u[C] + u[C + 1];
  const T d2p = u[C] - T(2.0) * u[C + 1] + u[C + 2];
  const T dm4jph = DM4(T(4.0) * d20 - d2p, T(4.0) * d2p - d20, d20, d2p);
  const T dm4jmh = DM4(T(4.0) * d20 - d2m, T(4.0) * d2m - d20, d20, d2m);
  const T vul = u[C] + alpha * du0;
  const T vav = T(0.5) * (u[C] + u[C + 1]);
  const T vmd = vav - T(0.5) * dm4jph;
  const T vlc = u[C] + T(0.5) * du0 + b2 * dm4jmh;
  const T vmin = fmax2(fmin2(fmin2(u[C], u[C + 1]), vmd), fmin2(fmin2(u[C], vul), vlc));
  const T vmax = fmin2(fmax2(fmax2(u[C], u[C + 1]), vmd), fmax2(fmax2(u[C], vul), vlc));
  return vorp + DMM(vmin - vorp, vmax - vorp);
}
template <int RM, int C, typename T, int N>
__device__ __forceinline__ T mp_up(const T (&u)[N]) {
  bool ok;
  const T v = mp_up_fast<RM, C>(u, ok);
  return ok ? v : mp_up_lim<RM, C>(u, v);
}

// um(k) for the cell at register index C (mp5.f95:142-167), same two steps
template <int RM, int C, typename T, int N>
__device__ __forceinline__ T mp_um_fast(const T (&u)[N], bool& ok) {
  const T alpha = T(2.0), epsm = T(1.0e-10);
  const T du0 = u[C] - u[C - 1];
  const T du1 = u[C + 1] - u[C];
  const T vorm = mp_vorm<RM, C>(u);
  const T vmpm = u[C] + DMM(-du0, -alpha * du1);
  ok = (vorm - u[C]) * (vorm - vmpm) <= epsm;
  return vorm;
}
template <int RM, int C, typename T, int N>
__device__ __forceinline__ T mp_um_lim(const T (&u)[N], T vorm) {
  const T alpha = T(2.0), b2 = T(4.0 / 3.0);
  const T du1 = u[C + 1] - u[C];
  const T d2m = u[C - 2] - T(2.0) * u[C - 1] + u[C];
  const T d20 = u[C - 1] - T(2.0) * u[C] + u[C + 1];
  const T d2p = u[C] - T(2.0) * u[C + 1] + u[C + 2];
  const T dm4jph = DM4(T(4.0) * d20 - d2p, T(4.0) * d2p - d20, d20, d2p);
  const T dm4jmh = DM4(T(4.0) * d20 - d2m, T(4.0) * d2m - d20, d20, d2m);
  const T vul = u[C] - alpha * du1;
  const T vav = T(0.5) * (u[C] + u[C - 1]);
  const T vmd = vav - T(0.5) * dm4jmh;
  const T vlc = u[C] - T(0.5) * du1 + b2 * dm4jph;
  const T vmin = fmax2(fmin2(fmin2(u[C], u[C - 1]), vmd), fmin2(fmin2(u[C], vul), vlc));
  const T vmax = fmin2(fmax2(fmax2(u[C], u[C - 1]), vmd), fmax2(fmax2(u[C], vul), vlc));
  return vorm + DMM(vmin - vorm, vmax - vorm);
}
template <int RM, int C, typename T, int N>
__device__ __forceinline__ T mp_um(const T (&u)[N]) {
  bool ok;
  const T v = mp_um_fast<RM, C>(u, ok);
  return ok ? v : mp_um_lim<RM, C>(u, v);
}

// interface pair: u holds cells i-R .. i+1+R; returns L = up(i), R = um(i+1)
// (both monotonicity tests first: two independent chains before the rare
// limiting steps)
template <int RM, typename T, int N>
__device__ __forceinline__ void mp_pair(const T (&u)[N], T& L, T& R) {
  constexpr int C = MPR<RM>::R;
  bool okL, okR;
  L = mp_up_fast<RM, C>(u, okL);
  R = mp_um_fast<RM, C + 1>(u, okR);
  if (!okL) L = mp_up_lim<RM, C>(u, L);
  if (!okR) R = mp_um_lim<RM, C + 1>(u, R);
}
// up(k), um(k) of the cells at C and C + 1 (the positivity-fixed pairs),
// the four tests first
template <int RM, int C, typename T, int N>
__device__ __forceinline__ void mp_quad(const T (&u)[N], T& up0, T& um0, T& up1, T& um1) {
  bool o0, o1, o2, o3;
  up0 = mp_up_fast<RM, C>(u, o0);
  um0 = mp_um_fast<RM, C>(u, o1);
  up1 = mp_up_fast<RM, C + 1>(u, o2);
  um1 = mp_um_fast<RM, C + 1>(u, o3);
  if (!o0) up0 = mp_up_lim<RM, C>(u, up0);
  if (!o1) um0 = mp_um_lim<RM, C>(u, um0);
  if (!o2) up1 = mp_up_lim<RM, C + 1>(u, up1);
  if (!o3) um1 = mp_um_lim<RM, C + 1>(u, um1);
}

// pair for the p / rho slots: the positivity fix-up of mp5.f95:177-216 makes
// the final up(k) depend on um(k) and the final um(k) on up(k)
template <typename T>
__device__ __forceinline__ void posfix_point(T uk, T duk, T duk1, T& up, T& um) {
  if (up < T(0.0)) { up = uk + T(0.50) * DMM(duk, duk1); um = uk; }
  if (um < T(0.0)) { um = uk - T(0.50) * DMM(duk, duk1); up = uk; }
}
template <int RM, typename T, int N>
__device__ __forceinline__ void mp_pair_pos(const T (&u)[N], T& L, T& R) {
  constexpr int C = MPR<RM>::R;
  T up0, um0, up1, um1;
  mp_quad<RM, C>(u, up0, um0, up1, um1);
  posfix_point(u[C], u[C] - u[C - 1], u[C + 1] - u[C], up0, um0);
  posfix_point(u[C + 1], u[C + 1] - u[C], u[C + 2] - u[C + 1], up1, um1);
  L = up0;
  R = um1;
}

// positivity-fixed pair on differences u - c0 (mixed precision): the same
// limiter (it is translation-equivariant) with the sign tests of the
// positivity fix taken on the FP64 value c0 + u
template <typename T>
__device__ __forceinline__ void posfix_point_delta(double c0, T uk, T duk, T duk1, T& up, T& um) {
  if (c0 + double(up) < 0.0) { up = uk + T(0.50) * DMM(duk, duk1); um = uk; }
  if (c0 + double(um) < 0.0) { um = uk - T(0.50) * DMM(duk, duk1); up = uk; }
}
template <int RM, typename T, int N>
__device__ __forceinline__ void mp_pair_pos_delta(const T (&u)[N], double c0, T& L, T& R) {
  constexpr int C = MPR<RM>::R;
  T up0, um0, up1, um1;
  mp_quad<RM, C>(u, up0, um0, up1, um1);
  posfix_point_delta(c0, u[C], u[C] - u[C - 1], u[C + 1] - u[C], up0, um0);
  posfix_point_delta(c0, u[C + 1], u[C + 1] - u[C], u[C + 2] - u[C + 1], up1, um1);
  L = up0;
  R = um1;
}

// Out-of-line entry points.  A sweep thread reconstructs ~45 slots per grid
// point; inlining the limiter 45 times made the kernel larger than the
// instruction cache (ncu: "no instruction" was the top stall).  One copy of
// each limiter body is called with the stencil values in registers.
template <typename T> struct Pair { T L, R; };

template <int RM, typename T> struct MPCall;
template <typename T> struct MPCall<0, T> {
  static __device__ __noinline__ Pair<T> pair(T a0, T a1, T a2, T a3, T a4, T a5) {
    const T u[6] = {a0, a1, a2, a3, a4, a5};
    Pair<T> p; mp_pair<0>(u, p.L, p.R); return p;
  }
  static __device__ __noinline__ Pair<T> pos(T a0, T a1, T a2, T a3, T a4, T a5) {
    const T u[6] = {a0, a1, a2, a3, a4, a5};
    Pair<T> p; mp_pair_pos<0>(u, p.L, p.R); return p;
  }
  static __device__ __noinline__ Pair<T> posd(T a0, T a1, T a2, T a3, T a4, T a5, double c0) {
    const T u[6] = {a0, a1, a2, a3, a4, a5};
    Pair<T> p; mp_pair_pos_delta<0>(u, c0, p.L, p.R); return p;
  }
  static __device__ __forceinline__ Pair<T> call_posd(const T (&u)[6], double c0) { return posd(u[0], u[1], u[2], u[3], u[4], u[5], c0); }
  template <bool POS> static __device__ __forceinline__ Pair<T> call(const T (&u)[6]) {
    return POS ? pos(u[0], u[1], u[2], u[3], u[4], u[5]) : pair(u[0], u[1], u[2], u[3], u[4], u[5]);
  }
};
template <typename T> struct MPCall<1, T> {
  static __device__ __noinline__ Pair<T> pair(T a0, T a1, T a2, T a3, T a4, T a5, T a6, T a7) {
    const T u[8] = {a0, a1, a2, a3, a4, a5, a6, a7};
    Pair<T> p; mp_pair<1>(u, p.L, p.R); return p;
  }
  static __device__ __noinline__ Pair<T> pos(T a0, T a1, T a2, T a3, T a4, T a5, T a6, T a7) {
    const T u[8] = {a0, a1, a2, a3, a4, a5, a6, a7};
    Pair<T> p; mp_pair_pos<1>(u, p.L, p.R); return p;
  }
  static __device__ __noinline__ Pair<T> posd(T a0, T a1, T a2, T a3, T a4, T a5, T a6, T a7, double c0) {
    const T u[8] = {a0, a1, a2, a3, a4, a5, a6, a7};
    Pair<T> p; mp_pair_pos_delta<1>(u, c0, p.L, p.R); return p;
  }
  static __device__ __forceinline__ Pair<T> call_posd(const T (&u)[8], double c0) { return posd(u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7], c0); }
  template <bool POS> static __device__ __forceinline__ Pair<T> call(const T (&u)[8]) {
    return POS ? pos(u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7])
               : pair(u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7]);
  }
};
template <typename T> struct MPCall<2, T> {
  static __device__ __noinline__ Pair<T> pair(T a0, T a1, T a2, T a3, T a4, T a5, T a6, T a7, T a8, T a9) {
    const T u[10] = {a0, a1, a2, a3, a4, a5, a6, a7, a8, a9};
    Pair<T> p; mp_pair<2>(u, p.L, p.R); return p;
  }
  static __device__ __noinline__ Pair<T> pos(T a0, T a1, T a2, T a3, T a4, T a5, T a6, T a7, T a8, T a9) {
    const T u[10] = {a0, a1, a2, a3, a4, a5, a6, a7, a8, a9};
    Pair<T> p; mp_pair_pos<2>(u, p.L, p.R); return p;
  }
  static __device__ __noinline__ Pair<T> posd(T a0, T a1, T a2, T a3, T a4, T a5, T a6, T a7, T a8, T a9, double c0) {
    const T u[10] = {a0, a1, a2, a3, a4, a5, a6, a7, a8, a9};
    Pair<T> p; mp_pair_pos_delta<2>(u, c0, p.L, p.R); return p;
  }
  static __device__ __forceinline__ Pair<T> call_posd(const T (&u)[10], double c0) { return posd(u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7], u[8], u[9], c0); }
  template <bool POS> static __device__ __forceinline__ Pair<T> call(const T (&u)[10]) {
    return POS ? pos(u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7], u[8], u[9])
               : pair(u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7], u[8], u[9]);
  }
};

// second-order MC pair of 16_hll_flow_mcl.f95:565-1112 (FAC = 0.5, no
// positivity fix): u holds cells i-1 .. i+2
template <typename T> struct MPCall<3, T> {
  template <bool POS> static __device__ __forceinline__ Pair<T> call(const T (&u)[4]) {
    Pair<T> p;
    p.L = u[1] + T(0.5) * mc_slope(u[2] - u[1], u[1] - u[0]);
    p.R = u[2] - T(0.5) * mc_slope(u[3] - u[2], u[2] - u[1]);
    return p;
  }
};

}  // namespace cueva
