// cueva_point.cuh -- pointwise physics of the CUEVA step, all FP64:
// startconvar (prim -> cons), the implicit Ohm's-law stage solve, the
// current J, the stiff source, and the two conserved-to-primitive solvers.
#pragma once
#include <math_constants.h>
#include "cueva_common.cuh"

namespace cueva {

// 06_conserved_var.f95:86-133
struct Cons { double D, tau, Sx, Sy, Sz, W; };
__device__ __forceinline__ Cons startconvar(double rho, double p, double vx, double vy, double vz,
                                            double Ex, double Ey, double Ez, double Bx, double By, double Bz,
                                            double gamma) {
  Cons c;
  const double V2 = pw2(vx) + pw2(vy) + pw2(vz);
  const double W = 1.0 / sqrt(1.0 - V2);
  const double E2 = pw2(Ex) + pw2(Ey) + pw2(Ez);
  const double B2 = pw2(Bx) + pw2(By) + pw2(Bz);
  const double eps = p / ((gamma - 1.0) * rho);
  const double h = rho * (1.0 + eps) + p;
  c.D = rho * W;
  c.tau = 0.5 * (E2 + B2) + h * pw2(W) - p;
  c.Sx = (Bz * Ey - By * Ez) + h * pw2(W) * vx;
  c.Sy = (Bx * Ez - Bz * Ex) + h * pw2(W) * vy;
  c.Sz = (By * Ex - Bx * Ey) + h * pw2(W) * vz;
  c.W = W;
  return c;
}

// 11_elecvarint.f95:289-323 (IMEX, REC_PRIM = 0): closed-form solve of
// E - E* = -a W (E + v x B - (E.v) v), a = Abt(l,l) sigma dt, with the
// time-n W, v and the stage-l B.
__device__ __forceinline__ void implicit_e(double abtll, double sigma, double dt, double W,
                                           double vx, double vy, double vz, double Bx, double By, double Bz,
                                           double Exa, double Eya, double Eza,
                                           double& Ex, double& Ey, double& Ez) {
  const double al = abtll * sigma * dt;
  const double matx = pw2(W) * al + W * pw2(al) + W + al;
  const double vrotB_x = (Bz * vy - By * vz);
  const double vrotB_y = (Bx * vz - Bz * vx);
  const double vrotB_z = (By * vx - Bx * vy);
  const double aW2 = al * pw2(W);
  const double cs = abtll * sigma * W * dt;
  const double mxx = al + W + aW2 * pw2(vx);
  const double myy = al + W + aW2 * pw2(vy);
  const double mzz = al + W + aW2 * pw2(vz);
  const double mxy = aW2 * vx * vy, mxz = aW2 * vx * vz, myz = aW2 * vy * vz;
  const double r = 1.0 / matx;
  Ex = r * (mxx * Exa + mxy * Eya + mxz * Eza - cs * (mxx * vrotB_x + mxy * vrotB_y + mxz * vrotB_z));
  Ey = r * (mxy * Exa + myy * Eya + myz * Eza - cs * (mxy * vrotB_x + myy * vrotB_y + myz * vrotB_z));
  Ez = r * (mxz * Exa + myz * Eya + mzz * Eza - cs * (mxz * vrotB_x + myz * vrotB_y + mzz * vrotB_z));
}

// 14_flowinit.f95:280-302: J = sigma W (E + v x B - (E.v) v) + q v
__device__ __forceinline__ void current(double sigma, double W, double vx, double vy, double vz,
                                        double Ex, double Ey, double Ez, double Bx, double By, double Bz,
                                        double q, double& Jx, double& Jy, double& Jz) {
  const double Edotv = Ex * vx + Ey * vy + Ez * vz;
  const double vrotB_x = (Bz * vy - By * vz);
  const double vrotB_y = (Bx * vz - Bz * vx);
  const double vrotB_z = (By * vx - Bx * vy);
  Jx = sigma * W * (Ex + vrotB_x - Edotv * vx) + q * vx;
  Jy = sigma * W * (Ey + vrotB_y - Edotv * vy) + q * vy;
  Jz = sigma * W * (Ez + vrotB_z - Edotv * vz) + q * vz;
}

// 17_fluxandsource.f95:529-536: stiff source with time-n W, v
__device__ __forceinline__ void stiff_source(double sigma, double W, double vx, double vy, double vz,
                                             double Ex, double Ey, double Ez, double Bx, double By, double Bz,
                                             double& Sx, double& Sy, double& Sz) {
  const double Edotv = Ex * vx + Ey * vy + Ez * vz;
  const double vrotB_x = (Bz * vy - By * vz);
  const double vrotB_y = (Bx * vz - Bz * vx);
  const double vrotB_z = (By * vx - Bx * vy);
  Sx = sigma * W * (Ex + vrotB_x - Edotv * vx);
  Sy = sigma * W * (Ey + vrotB_y - Edotv * vy);
  Sz = sigma * W * (Ez + vrotB_z - Edotv * vz);
}

struct C2PIn { double D, tau, Sx, Sy, Sz, Ex, Ey, Ez, Bx, By, Bz, vx0, vy0, vz0, rho0, p0; };
struct C2POut { double vx, vy, vz, rho, p, W; };

// pressure fixed-point ("pressure NR", epsilon frozen), 12_varprimitive.f95:558-587
__device__ __forceinline__ double frozen_eps_pressure(double p0, double rho, double eps, double V2c,
                                                      double gamma) {
  const double Cs2 = (gamma * (gamma - 1.0) * eps) / (1.0 + gamma * eps);
  double pnro = p0, CHA = 1.0;
  for (int nr = 1; CHA >= 1.0e-10 && nr <= 40; ++nr) {
    const double pnr = pnro - ((gamma - 1.0) * rho * eps - pnro) / (V2c * Cs2 - 1.0);
    CHA = fabs(pnr - pnro) / (0.5 * (pnr + pnro));
    pnro = pnr;
  }
  return pnro;
}

// velocities from S - E x B over tau - E2B2 + p (12_varprimitive.f95:615-624)
__device__ __forceinline__ void velocity_from_cons(const C2PIn& in, double tau, double E2B2, double p,
                                                   double& vx, double& vy, double& vz) {
  vx = (in.Sx - in.Ey * in.Bz + in.Ez * in.By) / (tau - E2B2 + p);
  vy = (in.Sy - in.Ez * in.Bx + in.Ex * in.Bz) / (tau - E2B2 + p);
  vz = (in.Sz - in.Ex * in.By + in.Ey * in.Bx) / (tau - E2B2 + p);
}

// Given W and rho, the pressure update, fix-ups and velocity recovery of
// 12_varprimitive.f95:533-696 (shared by Cardano and the learned-seed path).
__device__ __forceinline__ uint32_t c2p_finish(const C2PIn& in, double W_elec, double V2c0, double E2B2,
                                               double gamma, C2POut& o, unsigned long long* cnt) {
  uint32_t st = 0;
  const double gamma_1 = (gamma - 1.0) / gamma;
  double rho_elec = in.D / W_elec;
  if (rho_elec < 0.0) {
    if (cnt) atomicAdd(&cnt[0], 1ull);
    rho_elec = fmax2(in.rho0 * 1.0e-1, rho_elec);
  }
  double enthpy_elec = (in.tau - E2B2 - gamma_1 * rho_elec) / (pw2(W_elec) - gamma_1);
  double p_elec = gamma_1 * (enthpy_elec - rho_elec);
  const double epsilonnr = (in.tau - E2B2 - in.D * W_elec + p_elec * (1.0 - pw2(W_elec))) / (in.D * W_elec);
  double pnro = frozen_eps_pressure(p_elec, rho_elec, epsilonnr, V2c0, gamma);
  if (pnro < 0.0) {
    if (cnt) atomicAdd(&cnt[1], 1ull);
    pnro = fmax2(in.p0 * 1.0e-4, pnro);
  }
  p_elec = pnro;
  double tau_elec = E2B2 + enthpy_elec * pw2(W_elec) - p_elec;
  double vx, vy, vz;
  velocity_from_cons(in, tau_elec, E2B2, p_elec, vx, vy, vz);
  double V2c = pw2(vx) + pw2(vy) + pw2(vz);
  W_elec = 1.0 / sqrt(1.0 - V2c);
  if (V2c >= 1.0) {  // drift-velocity rescue, :627-696
    const double ErotB = in.Ey * in.Bz - in.Ez * in.By + in.Ez * in.Bx - in.Ex * in.Bz + in.Ex * in.By - in.Ey * in.Bx;
    const double B2_drift = pw2(in.Bx) + pw2(in.By) + pw2(in.Bz);
    if (B2_drift / rho_elec >= 10.0) {
      const double v_drift = ErotB / B2_drift;
      const double W_drift = 1.0 / sqrt(1.0 - pw2(v_drift));
      rho_elec = in.D / W_drift;
      enthpy_elec = (tau_elec - E2B2 - gamma_1 * rho_elec) / (pw2(W_drift) - gamma_1);
      p_elec = gamma_1 * (enthpy_elec - rho_elec);
      tau_elec = E2B2 + enthpy_elec * pw2(W_elec) - p_elec;
      velocity_from_cons(in, tau_elec, E2B2, p_elec, vx, vy, vz);
      V2c = pw2(vx) + pw2(vy) + pw2(vz);
      W_elec = 1.0 / sqrt(1.0 - V2c);
      if (cnt) atomicAdd(&cnt[2], 1ull);
      if (V2c >= 1.0) st |= ST_SUPERLUMINAL;
    } else {
      st |= ST_SUPERLUMINAL;
    }
  }
  o.vx = vx; o.vy = vy; o.vz = vz; o.rho = rho_elec; o.p = p_elec; o.W = W_elec;
  return st;
}

__device__ __forceinline__ double e2b2_half(const C2PIn& in) {
  return 0.5 * (pw2(in.Ex) + pw2(in.Ey) + pw2(in.Ez) + pw2(in.Bx) + pw2(in.By) + pw2(in.Bz));
}

// Cardano seed arithmetic with +,-,*,/ only, so host and device produce the
// same bits (the last bit of the W seed is amplified by the limiter switches
// of the reference scheme; libm-dependent acos/cos/pow would make CPU and GPU
// runs drift apart by ~1e-5 over 200 steps).
// Roots of 4c^3 - 3c = y, y in (-1, 1): by the triple-angle identity
// cos 3a = 4 cos^3 a - 3 cos a they are cos((acos y + 2 pi k)/3); c0 in
// (1/2, 1) and c1 in (-1, -1/2) by monotone Newton from c = 1 and c = -1,
// c2 from -(c0 + c1) (the roots sum to zero) polished by Newton.
__device__ __forceinline__ void chebyshev_roots(double y, double& c0, double& c1, double& c2) {
  double c = 1.0;
  for (int it = 0; it < 80; ++it) {
    const double cn = c - ((4.0 * c * c - 3.0) * c - y) / (12.0 * c * c - 3.0);
    if (!(cn < c)) break;
    c = cn;
  }
  c0 = c;
  c = -1.0;
  for (int it = 0; it < 80; ++it) {
    const double cn = c - ((4.0 * c * c - 3.0) * c - y) / (12.0 * c * c - 3.0);
    if (!(cn > c)) break;
    c = cn;
  }
  c1 = c;
  c = -(c0 + c1);
  for (int it = 0; it < 3; ++it) c = c - ((4.0 * c * c - 3.0) * c - y) / (12.0 * c * c - 3.0);
  c2 = c;
}
// x^(1/3), x >= 0: Newton cube root on the mantissa (frexp/ldexp are exact)
// d_2 + 2 z_1 under the square root of the one-real-root branch of
// 12_varprimitive.f95 vanishes where the depressed quartic is biquadratic
// (d_1 = 0), which the KH layer at V0 = 0.8 crosses at |v| ~ 0.74; there the
// sum is zero up to rounding and can come out as -1e-15, and the square root
// would return NaN with no status raised (the reference has no check on this
// branch).  A negative value within rounding of zero (<= 1e-12 |d_2|) is
// taken as zero, the biquadratic limit; anything else is left as it is.
__device__ __forceinline__ double biquad_guard(double s2, double d_2) {
  return (s2 < 0.0 && -s2 <= 1.0e-12 * fabs(d_2)) ? 0.0 : s2;
}

__device__ __forceinline__ double cbrt_newton(double x) {
  if (!(x > 0.0) || !(x < CUDART_INF)) return x;
  int e;
  double m = frexp(x, &e);
  const int r = ((e % 3) + 3) % 3;
  const int q = (e - r) / 3;
  m = ldexp(m, r);
  double y = 1.0;
#pragma unroll
  for (int it = 0; it < 8; ++it) y = y - (y * y * y - m) / (3.0 * y * y);
  return ldexp(y, q);
}

// Cardano con2prim, 12_varprimitive.f95:48-813 (l_swap = 1, VDRIFT = 0,
// low_vel = 0, REC_ELEC = 0): quartic in W by Ferrari-Cardano, Newton polish.
__device__ __forceinline__ uint32_t c2p_cardano(const C2PIn& in, double gamma, double eps1, C2POut& o,
                                                unsigned long long* cnt) {
  uint32_t st = 0;
  double V2c = pw2(in.vx0) + pw2(in.vy0) + pw2(in.vz0);
  if (V2c > 1.0) V2c = fmax2(-1.0 + eps1, fmin2(1.0 - eps1, V2c));
  const double E2B2 = e2b2_half(in);
  const double gamma_1 = (gamma - 1.0) / gamma;
  const double C_1 = pw2(in.Sx - in.Ey * in.Bz + in.Ez * in.By) + pw2(in.Sy - in.Ez * in.Bx + in.Ex * in.Bz) +
                     pw2(in.Sz - in.Ex * in.By + in.Ey * in.Bx);
  const double C_2 = in.tau - E2B2;
  const double a_4 = C_1 - pw2(C_2);
  const double a_3 = 2.0 * gamma_1 * C_2 * in.D;
  const double a_2 = pw2(C_2) - 2.0 * gamma_1 * C_1 - pw2(gamma_1) * pw2(in.D);
  const double a_1 = -2.0 * gamma_1 * C_2 * in.D;
  const double a_0 = pw2(gamma_1) * (C_1 + pw2(in.D));
  const double b_3 = a_3 / a_4, b_2 = a_2 / a_4, b_1 = a_1 / a_4, b_0 = a_0 / a_4;
  const double d_2 = b_2 - (3.0 * pw2(b_3)) / 8.0;
  const double d_1 = b_1 - (b_3 * b_2) / 2.0 + (pw3(b_3)) / 8.0;
  const double d_0 = b_0 - (b_3 * b_1) / 4.0 + (pw2(b_3) * b_2) / 16.0 - (3.0 * pw4(b_3)) / 256.0;
  const double e = (20.0 * d_2) / 8.0;
  const double f = -(d_0 - 2.0 * pw2(d_2));
  const double g = -(pw2(d_1) + 4.0 * d_2 * d_0 - 4.0 * pw3(d_2)) / 8.0;
  const double Q_1 = (pw2(e) - 3.0 * f) / 9.0;
  const double R_1 = (2.0 * pw3(e) - 9.0 * e * f + 27.0 * g) / 54.0;
  double s = 0.0, t = 0.0, det = 0.0, z_1 = 0.0;
  if (pw2(R_1) < pw3(Q_1)) {
    double ca, cb, cc;   // cos(T/3), cos((T+2pi)/3), cos((T-2pi)/3), T = acos(R/|Q|^1.5)
    chebyshev_roots(R_1 / fabs(sqrt(pw3(Q_1))), ca, cb, cc);
    const double sq = fabs(sqrt(Q_1));
    const double zs[3] = {-2.0 * sq * ca - e / 3.0, -2.0 * sq * cb - e / 3.0, -2.0 * sq * cc - e / 3.0};
    bool found = false;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      if (found) break;
      const double s_1 = d_2 + 2.0 * zs[r];
      const double t_1 = pw2(zs[r]) + 2.0 * d_2 * zs[r] + pw2(d_2) - d_0;
      if (s_1 >= 0.0 && t_1 >= 0.0) {
        s = fabs(sqrt(s_1));
        t = fabs(sqrt(t_1));
        det = pw2(s) - 4.0 * (d_2 + zs[r] - t);
        z_1 = zs[r];
        if (det < 0.0) st |= ST_C2P_FAIL;
        found = true;
      }
    }
    if (!found) st |= ST_C2P_FAIL;
  } else {
    const double xx1 = fabs(R_1) + fabs(sqrt(pw2(R_1) - pw3(Q_1)));
    const double AA_1 = -fsgn1(R_1) * copysign(fabs(cbrt_newton(xx1)), xx1);
    const double BB_1 = (AA_1 != 0.0) ? Q_1 / AA_1 : 0.0;
    z_1 = (AA_1 + BB_1) - e / 3.0;
    s = fabs(sqrt(biquad_guard(d_2 + 2.0 * z_1, d_2)));
    t = fabs(sqrt(pw2(z_1) + 2.0 * d_2 * z_1 + pw2(d_2) - d_0));
    det = pw2(s) - 4.0 * (d_2 + z_1 - t);
  }
  const double Q_2 = -0.5 * (-s + fsgn1(-s) * fabs(sqrt(det)));
  const double y_1 = Q_2 - b_3 / 4.0;
  const double y_2 = (d_2 + z_1 - t) / Q_2 - b_3 / 4.0;
  double Wnro = CUDART_NAN;
  if (y_1 >= 1.0 && y_2 >= 1.0) Wnro = fmin2(y_1, y_2);
  if (y_1 <= 1.0 && y_2 <= 1.0) st |= ST_C2P_FAIL;
  if (y_1 >= 1.0 && y_2 <= 1.0) Wnro = y_1;
  if (y_1 <= 1.0 && y_2 >= 1.0) Wnro = y_2;
  // Newton polish of W, 12_varprimitive.f95:510-526
  double CHA1 = 1.0;
  for (int nrw = 1; CHA1 > 1.0e-10 && nrw < 40; ++nrw) {
    const double Wnr = Wnro - (pw4(Wnro) + b_3 * pw3(Wnro) + b_2 * pw2(Wnro) + b_1 * Wnro + b_0) /
                              (4.0 * pw3(Wnro) + 3.0 * b_3 * pw2(Wnro) + 2.0 * b_2 * Wnro + b_1);
    CHA1 = fabs(Wnr - Wnro) / (0.5 * (Wnr + Wnro));
    Wnro = Wnr;
  }
  st |= c2p_finish(in, Wnro, V2c, E2B2, gamma, o, cnt);
  return st;
}

// Newton-Raphson con2prim, 12_varprimitive_nr.f95:28-338 (l_swap = 1)
__device__ __forceinline__ uint32_t c2p_nr(const C2PIn& in, double gamma, C2POut& o) {
  uint32_t st = 0;
  const double E2B2 = e2b2_half(in);
  double p_elec = in.p0;
  double vx, vy, vz;
  velocity_from_cons(in, in.tau, E2B2, p_elec, vx, vy, vz);
  double V2c = pw2(vx) + pw2(vy) + pw2(vz);
  double W = 1.0 / sqrt(1.0 - V2c);
  double W_2 = 1.0 / (1.0 - V2c);
  double rho = in.D / W;
  const double epsilonnr = (in.tau - E2B2 - in.D * W + p_elec * (1.0 - W_2)) / (in.D * W);
  p_elec = frozen_eps_pressure(p_elec, rho, epsilonnr, V2c, gamma);
  velocity_from_cons(in, in.tau, E2B2, p_elec, vx, vy, vz);
  V2c = pw2(vx) + pw2(vy) + pw2(vz);
  W = 1.0 / sqrt(1.0 - V2c);
  rho = in.D / W;
  if (V2c >= 1.0) st |= ST_SUPERLUMINAL;
  o.vx = vx; o.vy = vy; o.vz = vz; o.rho = rho; o.p = p_elec; o.W = W;
  return st;
}

}  // namespace cueva
