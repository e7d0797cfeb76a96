// cueva_diag.cu -- device-side reductions of the run diagnostics: the volume
// integrals and maxima that the reference's writer accumulates after every
// hglb-th step (22_writer.f95:821-1001, subroutine lector, DIM == 2), plus a
// Courant-number check (largest |v|, Lorentz factor and sound-wave speed).
//
// Two launches: every CTA reduces a fixed set of points into one row of
// partial results (warp shuffles, then the CTA's warps in order), and one CTA
// combines the rows in CTA order and writes a record.  The point set of each
// thread and every combination order depend only on the grid size, so a
// record is bit-reproducible from run to run; its sums differ from the
// reference's left-to-right loop only by summation rounding.
#include <cmath>
#include "cueva_launch.h"
#include "../../include/cueva.h"

namespace cueva {
namespace {

constexpr int DG_THREADS = 256;
constexpr int DG_NSUM = 35;            // sums, record slots 0..34
constexpr int DG_NMAX = 6;             // maxima: Bx/B0, phi, |v|, W, |lambda_x|, |lambda_y|
constexpr int DG_NPART = DG_NSUM + DG_NMAX;
static_assert(CUEVA_DG_SUM_D_MED + 1 == DG_NSUM, "record slots 0..34 are the sums");

struct DiagArgs {
  const double* prim;   // 14 primitive slabs
  const double* D;      // conserved D and tau slabs at the time of the record
  const double* tau;
  int imax, jmax, pitch;
  long long fs;
  int imed1, imed2;     // floor(0.25 imax), floor(0.75 imax)
  double delx, dely, gamma, b0;
};

// largest |lambda| of the two relativistic sound waves along direction n
// (normal velocity vn, V2 = v.v, cs2 = gamma p / (rho h) with the enthalpy
// density rho h = rho (1 + eps) + p)
template <typename R>
__host__ __device__ inline R sound_lambda(R vn, R V2, R cs2) {
  const R cs = sqrt(cs2);
  const R root = sqrt((R(1) - V2) * (R(1) - V2 * cs2 - vn * vn * (R(1) - cs2)));
  const R den = R(1) - cs2 * V2;
  const R lp = (vn * (R(1) - cs2) + cs * root) / den;
  const R lm = (vn * (R(1) - cs2) - cs * root) / den;
  return fmax(fabs(lp), fabs(lm));
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__global__ void __launch_bounds__(DG_THREADS) k_diag_partial(DiagArgs a, double* __restrict__ part) {
  const int nx = a.imax + 1;
  const long long npts = (long long)nx * (a.jmax + 1);
  const double dx = a.delx, dy = a.dely;
  double s[DG_NSUM];
#pragma unroll
  for (int k = 0; k < DG_NSUM; ++k) s[k] = 0.0;
  double m[DG_NMAX];
#pragma unroll
  for (int k = 0; k < DG_NMAX; ++k) m[k] = -INFINITY;
  const long long fs = a.fs;
  for (long long t = blockIdx.x * (long long)DG_THREADS + threadIdx.x; t < npts;
       t += (long long)gridDim.x * DG_THREADS) {
    const int i = int(t % nx), j = int(t / nx);
    const long long pc = (long long)j * a.pitch + i;
    const double* p = a.prim;
    const double rho = p[P_RHO * fs + pc], pr = p[P_P * fs + pc];
    const double vx = p[P_VX * fs + pc], vy = p[P_VY * fs + pc], vz = p[P_VZ * fs + pc];
    const double psi = p[P_PSI * fs + pc], phi = p[P_PHI * fs + pc];
    const double Ex = p[P_EX * fs + pc], Ey = p[P_EY * fs + pc], Ez = p[P_EZ * fs + pc];
    const double Bx = p[P_BX * fs + pc], By = p[P_BY * fs + pc], Bz = p[P_BZ * fs + pc];
    const double q = p[P_Q * fs + pc];
    const double D = a.D[pc], tau = a.tau[pc];
    // each term as the writer evaluates it: x * Delx * Dely, left to right
    s[CUEVA_DG_SUM_PSI] += (psi * dx) * dy;
    s[CUEVA_DG_SUM_PHI] += (phi * dx) * dy;
    s[CUEVA_DG_SUM_EX] += ((Ex * Ex) * dx) * dy;
    s[CUEVA_DG_SUM_EY] += ((Ey * Ey) * dx) * dy;
    s[CUEVA_DG_SUM_EZ] += ((Ez * Ez) * dx) * dy;
    s[CUEVA_DG_SUM_EXEY] += ((Ex * Ey) * dx) * dy;
    s[CUEVA_DG_SUM_EXEZ] += ((Ex * Ez) * dx) * dy;
    s[CUEVA_DG_SUM_EYEZ] += ((Ey * Ez) * dx) * dy;
    s[CUEVA_DG_SUM_BX] += ((Bx * Bx) * dx) * dy;
    s[CUEVA_DG_SUM_BY] += ((By * By) * dx) * dy;
    s[CUEVA_DG_SUM_BZ] += ((Bz * Bz) * dx) * dy;
    s[CUEVA_DG_SUM_BXBY] += ((Bx * By) * dx) * dy;
    s[CUEVA_DG_SUM_BXBZ] += ((Bx * Bz) * dx) * dy;
    s[CUEVA_DG_SUM_BYBZ] += ((By * Bz) * dx) * dy;
    const double B2all = (Bx * Bx + By * By) + Bz * Bz;
    const double V2 = (vx * vx + vy * vy) + vz * vz;
    s[CUEVA_DG_SUM_BXBYBZ] += (B2all * dx) * dy;
    s[CUEVA_DG_SUM_VXVYVZ] += (V2 * dx) * dy;
    s[CUEVA_DG_SUM_VX] += ((vx * vx) * dx) * dy;
    s[CUEVA_DG_SUM_VY] += ((vy * vy) * dx) * dy;
    s[CUEVA_DG_SUM_VZ] += ((vz * vz) * dx) * dy;
    s[CUEVA_DG_SUM_VXVY] += ((vx * vy) * dx) * dy;
    s[CUEVA_DG_SUM_VXVZ] += ((vx * vz) * dx) * dy;
    s[CUEVA_DG_SUM_VYVZ] += ((vy * vz) * dx) * dy;
    s[CUEVA_DG_SUM_Q] += (q * dx) * dy;
    s[CUEVA_DG_SUM_P] += (pr * dx) * dy;
    s[CUEVA_DG_SUM_RHO] += (rho * dx) * dy;
    s[CUEVA_DG_SUM_D] += (D * dx) * dy;
    if (i >= a.imed1 && i <= a.imed2) s[CUEVA_DG_SUM_D_MED] += (D * dx) * dy;
    const double eps = pr / ((a.gamma - 1.0) * rho);
    const double hh = rho * (1.0 + eps) + pr;
    const double W = 1.0 / sqrt(1.0 - V2);
    const double E2 = (Ex * Ex + Ey * Ey) + Ez * Ez;
    const double B2 = By * By + Bz * Bz;   // the writer's B2 leaves Bx out
    s[CUEVA_DG_EKIN_C] += (((0.5 * rho) * V2) * dx) * dy;
    s[CUEVA_DG_EKIN_R] += ((D * (W - 1.0)) * dx) * dy;
    s[CUEVA_DG_EINT_C] += ((rho * eps) * dx) * dy;
    // eint_r and efluid_r: only the p term carries Delx * Dely (operator
    // precedence of the writer's expressions), and the sum adds, then subtracts
    s[CUEVA_DG_EINT_R] = (s[CUEVA_DG_EINT_R] + (W * W) * (rho * eps + pr)) - (pr * dx) * dy;
    s[CUEVA_DG_ETOT] += (tau * dx) * dy;
    s[CUEVA_DG_EFLUID_R] = (s[CUEVA_DG_EFLUID_R] + hh * (W * W)) - (pr * dx) * dy;
    s[CUEVA_DG_EMAG] += ((0.5 * (E2 + B2)) * dx) * dy;
    s[CUEVA_DG_LORENTZ] += (W * dx) * dy;
    m[0] = fmax(m[0], Bx / a.b0);
    m[1] = fmax(m[1], phi);
    m[2] = fmax(m[2], sqrt(V2));
    m[3] = fmax(m[3], W);
    const double cs2 = a.gamma * pr / hh;
    m[4] = fmax(m[4], sound_lambda(vx, V2, cs2));
    m[5] = fmax(m[5], sound_lambda(vy, V2, cs2));
  }
  // CTA reduction: shuffle tree inside each warp, then warps in order
  __shared__ double sh[DG_THREADS / 32][DG_NPART];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < DG_NSUM; ++k) {
    const double v = warp_sum(s[k]);
    if (lane == 0) sh[w][k] = v;
  }
#pragma unroll
  for (int k = 0; k < DG_NMAX; ++k) {
    const double v = warp_max(m[k]);
    if (lane == 0) sh[w][DG_NSUM + k] = v;
  }
  __syncthreads();
  if (threadIdx.x < DG_NPART) {
    const int k = threadIdx.x;
    double v = sh[0][k];
    for (int ww = 1; ww < DG_THREADS / 32; ++ww) v = (k < DG_NSUM) ? v + sh[ww][k] : fmax(v, sh[ww][k]);
    part[(long long)blockIdx.x * DG_NPART + k] = v;
  }
}

__global__ void k_diag_final(DiagArgs a, const double* __restrict__ part, int nblk, long long h, double t,
                             double dt, cueva_diag_record* __restrict__ rec) {
  __shared__ double v[DG_NPART];
  const int k = threadIdx.x;
  if (k < DG_NPART) {
    double x = part[k];
    for (int b = 1; b < nblk; ++b) {
      const double y = part[(long long)b * DG_NPART + k];
      x = (k < DG_NSUM) ? x + y : fmax(x, y);
    }
    v[k] = x;
  }
  __syncthreads();
  if (k < DG_NSUM) rec->v[k] = v[k];
  if (k == 0) {
    rec->h = h;
    rec->t = t;
    rec->v[CUEVA_DG_MAX_BX] = v[DG_NSUM + 0];
    rec->v[CUEVA_DG_MAX_PHI] = v[DG_NSUM + 1];
    rec->v[CUEVA_DG_MAX_V] = v[DG_NSUM + 2];
    rec->v[CUEVA_DG_MAX_W] = v[DG_NSUM + 3];
    rec->v[CUEVA_DG_MAX_LAMBDA_X] = v[DG_NSUM + 4];
    rec->v[CUEVA_DG_MAX_LAMBDA_Y] = v[DG_NSUM + 5];
    rec->v[CUEVA_DG_COURANT] = fmax(dt * (v[DG_NSUM + 4] / a.delx), dt * (v[DG_NSUM + 5] / a.dely));
    // point values of the reconnection-rate outputs (writer units 67, 68):
    // Ez(imed, jmed) and By(imed + 1, jmed + 1), imed = floor(imax / 2)
    const int imed = a.imax / 2, jmed = a.jmax / 2;
    const long long fs = a.fs;
    rec->v[CUEVA_DG_EZ_MED] = a.prim[P_EZ * fs + (long long)jmed * a.pitch + imed];
    const int i1 = imed + 1 <= a.imax ? imed + 1 : a.imax, j1 = jmed + 1 <= a.jmax ? jmed + 1 : a.jmax;
    rec->v[CUEVA_DG_BY_MED] = a.prim[P_BY * fs + (long long)j1 * a.pitch + i1];
    rec->v[CUEVA_DG_DELTA_REC] = 0.0;   // the host evaluates tanh and fills it on read
  }
}

}  // namespace

int diag_blocks(int imax, int jmax) {
  const long long npts = (long long)(imax + 1) * (jmax + 1);
  long long b = (npts + DG_THREADS - 1) / DG_THREADS;
  if (b > 148 * 4) b = 148 * 4;
  return (int)(b < 1 ? 1 : b);
}
int diag_partials() { return DG_NPART; }

cudaError_t launch_diag(const InstDesc& I, int cur, const double* D, const double* tau, double b0, double* part,
                        long long h, double t, cueva_diag_record* rec, cudaStream_t st) {
  DiagArgs a;
  a.prim = I.prim[cur];
  a.D = D;
  a.tau = tau;
  a.imax = I.imax; a.jmax = I.jmax; a.pitch = I.pitch; a.fs = I.fstride;
  a.imed1 = (int)std::floor(0.25 * I.imax);
  a.imed2 = (int)std::floor(0.75 * I.imax);
  a.delx = I.delx; a.dely = I.dely; a.gamma = I.gamma;
  a.b0 = b0;
  const int nblk = diag_blocks(I.imax, I.jmax);
  k_diag_partial<<<nblk, DG_THREADS, 0, st>>>(a, part);
  k_diag_final<<<1, 64, 0, st>>>(a, part, nblk, h, t, I.dt, rec);
  return cudaGetLastError();
}

}  // namespace cueva
