// cueva_mlp.cuh -- learned con2prim seed: a 6 -> 64 -> 64 -> 64 -> 1 SiLU
// network predicts log p from the conserved state, a Newton-Raphson solve of
// the exact pressure equation refines it, and the reference's Cardano
// recovery is the fallback whenever the refinement fails.
//
// Features: the six inputs D, |S|, tau, |B|^2, |E|^2 and S.B/(|S||B|),
// normalised with the physics of the inversion.  With the fluid momentum
// Sf = S - E x B, the fluid energy Ef = tau - (E^2+B^2)/2 and
// M = sqrt(Ef^2 - |Sf|^2) (= W sqrt(rho h (rho h - 2p)) + O(p^2)):
//   f0 = log D,  f1 = log(Ef / M) (~ log W),  f2 = log(M/D - 1) (~ log 3p/rho),
//   f3 = log(1 + |B|^2/D),  f4 = log(1 + |E|^2/D),  f5 = S.B / (|S||B|);
// f2 carries the pressure through the cancellation M/D - 1, which plain
// log-scaled inputs lose (a network on log D, log(1 + |S|/D), log(tau/D), ...
// plateaus near a normalised MSE of 0.14 on the training set; this one
// reaches ~1e-4).  Each feature is normalised by the training set's mean and
// deviation; the output is the normalised log(p/D).  Weights are bf16,
// accumulation FP32.
//
// Pressure equation (ideal gas, h = rho + gamma/(gamma-1) p): with the
// fluid momentum Sf = S - E x B, the fluid energy Ef = tau - (E^2+B^2)/2 and
// Q = Ef + p = rho h W^2,
//   v^2 = |Sf|^2 / Q^2,   rho = D sqrt(1 - v^2),   rho h = Q (1 - v^2),
//   f(p) = p - (gamma-1)/gamma (rho h - rho) = 0,
//   f'(p) = 1 - (gamma-1)/gamma (1 + v^2 - D v^2 / (Q sqrt(1 - v^2))).
#pragma once
#include <cuda_bf16.h>
#include "cueva_point.cuh"

namespace cueva {

constexpr int MLP_IN = 6;
constexpr int MLP_H = 64;
// flat FP32 parameter vector: W1[64][6] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64] b4
constexpr int MLP_OFF_W1 = 0;
constexpr int MLP_OFF_B1 = MLP_OFF_W1 + MLP_H * MLP_IN;
constexpr int MLP_OFF_W2 = MLP_OFF_B1 + MLP_H;
constexpr int MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H;
constexpr int MLP_OFF_W3 = MLP_OFF_B2 + MLP_H;
constexpr int MLP_OFF_B3 = MLP_OFF_W3 + MLP_H * MLP_H;
constexpr int MLP_OFF_W4 = MLP_OFF_B3 + MLP_H;
constexpr int MLP_OFF_B4 = MLP_OFF_W4 + MLP_H;
constexpr int MLP_NPARAM = MLP_OFF_B4 + 1;            // 8833
constexpr int MLP_NNORM = 2 * MLP_IN + 2;              // feature mean/sd, target mean/sd
constexpr int MLP_NR_MAXIT = 30;

// network as the kernels read it (built from the FP32 master parameters)
struct MLPDevice {
  __nv_bfloat16 W1[MLP_H * MLP_IN];
  __nv_bfloat16 W2[MLP_H * MLP_H];
  __nv_bfloat16 W3[MLP_H * MLP_H];
  __nv_bfloat16 W4[MLP_H];
  float b1[MLP_H], b2[MLP_H], b3[MLP_H], b4;
  float mu[MLP_IN], sd[MLP_IN], mu_y, sd_y;
  unsigned long long* stats;   // [0] Newton iterations, [1] points, [2] Cardano fall-backs
};

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }

// raw (unnormalised) features of a conserved state (double arithmetic for
// the cancellations, rounded to float at the end)
__device__ __forceinline__ void c2p_features(double D, double tau, double Sx, double Sy, double Sz, double Ex,
                                             double Ey, double Ez, double Bx, double By, double Bz, float f[MLP_IN]) {
  const double S2 = Sx * Sx + Sy * Sy + Sz * Sz, B2 = Bx * Bx + By * By + Bz * Bz;
  const double E2 = Ex * Ex + Ey * Ey + Ez * Ez, SB = Sx * Bx + Sy * By + Sz * Bz;
  const double Sfx = Sx - (Ey * Bz - Ez * By), Sfy = Sy - (Ez * Bx - Ex * Bz), Sfz = Sz - (Ex * By - Ey * Bx);
  const double sfm = sqrt(Sfx * Sfx + Sfy * Sfy + Sfz * Sfz);
  const double Ef = tau - 0.5 * (E2 + B2);
  const double M = sqrt(fmax((Ef - sfm) * (Ef + sfm), 0.0));
  const double den = sqrt(S2 * B2);
  f[0] = (float)log(D);
  f[1] = (float)fmin(log(Ef / fmax(M, 1.0e-300)), 10.0);
  f[2] = (float)log(fmax(M / D - 1.0, 1.0e-9));
  f[3] = (float)log1p(B2 / D);
  f[4] = (float)log1p(E2 / D);
  f[5] = den > 0.0 ? (float)(SB / den) : 0.0f;
}

// normalised log(p/D) predicted for one state (one thread, FP32 FMA)
__device__ __forceinline__ float mlp_forward(const MLPDevice& M, const float f[MLP_IN]) {
  float x[MLP_IN];
#pragma unroll
  for (int k = 0; k < MLP_IN; ++k) x[k] = (f[k] - M.mu[k]) / M.sd[k];
  float a[MLP_H], b[MLP_H];
#pragma unroll 4
  for (int o = 0; o < MLP_H; ++o) {
    float z = M.b1[o];
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) z = fmaf(__bfloat162float(M.W1[o * MLP_IN + k]), x[k], z);
    a[o] = silu(z);
  }
#pragma unroll 2
  for (int o = 0; o < MLP_H; ++o) {
    float z = M.b2[o];
#pragma unroll
    for (int k = 0; k < MLP_H; ++k) z = fmaf(__bfloat162float(M.W2[o * MLP_H + k]), a[k], z);
    b[o] = silu(z);
  }
#pragma unroll 2
  for (int o = 0; o < MLP_H; ++o) {
    float z = M.b3[o];
#pragma unroll
    for (int k = 0; k < MLP_H; ++k) z = fmaf(__bfloat162float(M.W3[o * MLP_H + k]), b[k], z);
    a[o] = silu(z);
  }
  float y = M.b4;
#pragma unroll
  for (int k = 0; k < MLP_H; ++k) y = fmaf(__bfloat162float(M.W4[k]), a[k], y);
  return y;
}

// pressure seed of the network for a conserved state
__device__ __forceinline__ double mlp_pressure_seed(const MLPDevice& M, const C2PIn& in) {
  float f[MLP_IN];
  c2p_features(in.D, in.tau, in.Sx, in.Sy, in.Sz, in.Ex, in.Ey, in.Ez, in.Bx, in.By, in.Bz, f);
  const float y = mlp_forward(M, f) * M.sd_y + M.mu_y;
  return in.D * exp((double)y);
}

// Newton-Raphson on f(p) from the seed p; returns the iterations used, or
// -1 when the solve fails (non-finite, v >= 1, p <= 0, no convergence)
__device__ __forceinline__ int c2p_newton(const C2PIn& in, double gamma, double p, C2POut& o) {
  const double g1 = (gamma - 1.0) / gamma;
  const double Sfx = in.Sx - in.Ey * in.Bz + in.Ez * in.By;
  const double Sfy = in.Sy - in.Ez * in.Bx + in.Ex * in.Bz;
  const double Sfz = in.Sz - in.Ex * in.By + in.Ey * in.Bx;
  const double Sf2 = Sfx * Sfx + Sfy * Sfy + Sfz * Sfz;
  const double Ef = in.tau - e2b2_half(in);
  int it = 0;
  bool done = false;
  for (it = 1; it <= MLP_NR_MAXIT; ++it) {
    const double Q = Ef + p;
    const double v2 = Sf2 / (Q * Q);
    if (!(v2 < 1.0) || !(Q > 0.0)) return -1;
    const double sq = sqrt(1.0 - v2);
    const double f = p - g1 * (Q * (1.0 - v2) - in.D * sq);
    const double df = 1.0 - g1 * (1.0 + v2 - in.D * v2 / (Q * sq));
    const double dp = f / df;
    p -= dp;
    if (!(fabs(dp) > 1.0e-12 * fabs(p))) { done = true; break; }
  }
  if (!done || !(p > 0.0)) return -1;
  const double Q = Ef + p;
  const double v2 = Sf2 / (Q * Q);
  if (!(v2 < 1.0)) return -1;
  o.vx = Sfx / Q; o.vy = Sfy / Q; o.vz = Sfz / Q;
  o.W = 1.0 / sqrt(1.0 - v2);
  o.rho = in.D / o.W;
  o.p = p;
  return it;
}

// c2p method 2: network seed + Newton; Cardano when the refinement fails or
// no network is attached.  Out of line, so the network's 128 live FP32
// activations do not raise the register allocation of the kernels that
// merely contain this call.
static __device__ __noinline__ uint32_t c2p_learned(const C2PIn& in, double gamma, double eps1, const void* mlp,
                                                C2POut& o, unsigned long long* cnt) {
  if (!mlp) return c2p_cardano(in, gamma, eps1, o, cnt);
  const MLPDevice& M = *static_cast<const MLPDevice*>(mlp);
  const int it = c2p_newton(in, gamma, mlp_pressure_seed(M, in), o);
  if (M.stats) {
    // one atomic per warp and counter
    const unsigned mask = __activemask();
    const unsigned its = __reduce_add_sync(mask, (unsigned)(it > 0 ? it : MLP_NR_MAXIT));
    const unsigned nfail = __reduce_add_sync(mask, it > 0 ? 0u : 1u);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(mask) - 1)) {
      atomicAdd(&M.stats[0], (unsigned long long)its);
      atomicAdd(&M.stats[1], (unsigned long long)__popc(mask));
      if (nfail) atomicAdd(&M.stats[2], (unsigned long long)nfail);
    }
  }
  if (it > 0) return 0u;
  return c2p_cardano(in, gamma, eps1, o, cnt);
}

}  // namespace cueva
