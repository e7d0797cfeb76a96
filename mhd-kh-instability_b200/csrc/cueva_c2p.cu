// cueva_c2p.cu -- con2prim with the learned seed on the tcgen05 tensor cores,
// as a kernel of its own after the last RK stage.
//
// With the learned method the last stage's update stops after varfin: it
// stores the new psi, phi, E, B, q as primitives and the evolved D, tau, S
// in the (consumed) final-sum slabs.  k_c2p_step then recovers rho, p, v in
// tiles of 128 points -- network seed on the tensor cores (cueva_mlp_tc.cuh),
// Newton-Raphson in FP64, the reference's Cardano recovery when Newton fails
// -- and runs the next step's startconvar and stage-1 preparation, exactly
// as the fused epilogue does for the other methods.  Keeping the network
// out of the stencil kernel leaves that kernel's registers and occupancy
// alone and lets the network run at tensor-core rate with its weights
// staged once per CTA.
#include "cueva_launch.h"
#include "cueva_mlp_tc.cuh"
#include "cueva_stage.cuh"

namespace cueva {
namespace {

constexpr int C2P_CTAS_PER_SM = 4;
// k_c2p_step holds a tile's inputs in registers while it works on the one
// before: three CTAs per SM leave it the registers for that
constexpr int C2P_STEP_CTAS_PER_SM = 3;

// one point of the learned con2prim (all 128 threads of the CTA call it, in
// step): seeds p from the previous pressure or the network (the one with the
// smaller residual), refines it, falls back to Cardano
struct LearnedOut {
  C2POut o;
  uint32_t st;
  int it;
};
__device__ __forceinline__ bool learned_point(MLPShared& S, uint32_t& phase, const C2PIn& in, double gamma,
                                              double eps1, unsigned long long* counters, bool count, LearnedOut& r) {
  // The network's seeds leave Newton about 1e-2 from the root.  Where the
  // previous pressure is already closer than that for every point of the
  // tile (residual <= 1e-2 p), the tile skips the network; otherwise the
  // tile runs it and each point starts from the better of the two seeds.
  const double r_prev = c2p_residual(in, gamma, in.p0);
  double seed = in.p0;
  if (!__syncthreads_and(r_prev <= 1.0e-2 * in.p0)) {   // uniform over the CTA (one tile)
    float f[MLP_IN];
    c2p_features(in.D, in.tau, in.Sx, in.Sy, in.Sz, in.Ex, in.Ey, in.Ez, in.Bx, in.By, in.Bz, f);
    float y = 0.0f;
    if (!mlp_tc_tile(S, phase, f, y)) return false;
    const double p_net = in.D * (double)__expf(y * S.sd_y + S.mu_y);
    seed = c2p_residual(in, gamma, p_net) < r_prev ? p_net : in.p0;
  }
  r.it = c2p_newton(in, gamma, seed, r.o);
  r.st = 0u;
  if (r.it <= 0) r.st = c2p_cardano_ool(in, gamma, eps1, r.o, count ? counters : nullptr);
  if (!(isfinite(r.o.rho) && isfinite(r.o.p) && isfinite(r.o.vx) && isfinite(r.o.vy) && isfinite(r.o.vz)))
    r.st |= ST_NONFINITE;
  return true;
}

// Newton iterations, points and Cardano fall-backs: one atomic per warp and counter
__device__ __forceinline__ void learned_stats(unsigned long long* stats, bool count, int it) {
  if (!stats) return;
  const unsigned its = __reduce_add_sync(0xffffffffu, count ? (unsigned)(it > 0 ? it : MLP_NR_MAXIT) : 0u);
  const unsigned pts = __reduce_add_sync(0xffffffffu, count ? 1u : 0u);
  const unsigned nfail = __reduce_add_sync(0xffffffffu, (count && it <= 0) ? 1u : 0u);
  if ((threadIdx.x & 31) == 0) {
    if (pts) { atomicAdd(&stats[0], (unsigned long long)its); atomicAdd(&stats[1], (unsigned long long)pts); }
    if (nfail) atomicAdd(&stats[2], (unsigned long long)nfail);
  }
}

// L2 prefetch of the inputs of tile b of instance I (the 19 fields the
// tile reads; its 128 points cover at most two row segments per field)
__device__ __forceinline__ void c2p_prefetch(const InstDesc& I, int b, int cur) {
  const int t = threadIdx.x;
  if (t >= 2 * 19) return;
  const int nx = I.imax + 1;
  const long long npts = (long long)nx * (I.jmax + 1);
  const long long p0 = (long long)b * TC_ROWS;
  if (p0 >= npts) return;
  const long long p1 = (p0 + TC_ROWS < npts ? p0 + TC_ROWS : npts) - 1;   // last point of the tile
  const int f = t >> 1, seg = t & 1;
  const int j0 = int(p0 / nx), i0 = int(p0 % nx), j1 = int(p1 / nx), i1 = int(p1 % nx);
  if (seg == 1 && j1 == j0) return;
  const int row = seg ? j1 : j0, ia = seg ? 0 : i0, ib = (seg || j1 == j0) ? i1 : nx - 1;
  const long long fs = I.fstride;
  const double* base;
  if (f < 5) base = I.finsum + (long long)(Q_D + f) * fs;                   // varfin's D, tau, S
  else if (f < 14) base = I.prim[1 - cur] + (long long)(P_PSI + f - 5) * fs; // psi .. q of time n+1
  else base = I.prim[cur] + (long long)(f - 14) * fs;                       // rho, p, v seeds
  prefetch_l2(base + (long long)row * I.pitch + ia, ib - ia + 1);
}

// One thread's inputs of a tile: the con2prim state and the time n+1
// fields that varfin completed.  k_c2p_step loads them a tile ahead, so
// that their latency is spent under the previous tile's work.
struct C2PTileIn {
  C2PIn in;
  double fn[NPRIM - P_PSI];   // psi .. q of time n+1
  long long pc;               // the point's offset in its instance's slabs
  const InstDesc* I;
  int b;                      // the tile within its instance
  bool valid;                 // a real point (rows past the end repeat the last one)
  bool use;                   // the instance runs the learned method on the tensor cores
};

__device__ __forceinline__ void c2p_load(const InstDesc* __restrict__ insts, int ninst, int tile, int cur,
                                         C2PTileIn& t) {
  int b = tile;
  const InstDesc& I = tile_inst(insts, ninst, LK_C2P, b);
  t.I = &I;
  t.b = b;
  t.use = I.c2p == 2 && I.c2p_tc;   // uniform over the CTA: a tile belongs to one instance
  if (!t.use) return;
  const int nx = I.imax + 1;
  const long long npts = (long long)nx * (I.jmax + 1);
  const long long p0 = (long long)b * TC_ROWS + threadIdx.x;
  t.valid = p0 < npts;
  const long long p = t.valid ? p0 : npts - 1;
  const int i = int(p % nx), j = int(p / nx);
  const long long fs = I.fstride, pc = (long long)j * I.pitch + i;
  t.pc = pc;
  const double* un = I.finsum;        // varfin's D, tau, S in the slabs Q_D .. Q_SZ
  const double* pold = I.prim[cur];
  const double* pn = I.prim[1 - cur];
  t.in = C2PIn{un[Q_D * fs + pc], un[Q_TAU * fs + pc], un[Q_SX * fs + pc], un[Q_SY * fs + pc],
               un[Q_SZ * fs + pc], pn[P_EX * fs + pc], pn[P_EY * fs + pc], pn[P_EZ * fs + pc],
               pn[P_BX * fs + pc], pn[P_BY * fs + pc], pn[P_BZ * fs + pc], pold[P_VX * fs + pc],
               pold[P_VY * fs + pc], pold[P_VZ * fs + pc], pold[P_RHO * fs + pc], pold[P_P * fs + pc]};
#pragma unroll
  for (int c = P_PSI; c < NPRIM; ++c) t.fn[c - P_PSI] = pn[c * fs + pc];
}

// the tail of the step for the instances with the learned method: tiles of
// 128 points over all instances (block ranges of launch kind LK_C2P)
__global__ void __launch_bounds__(TC_ROWS, C2P_STEP_CTAS_PER_SM)
k_c2p_step(const InstDesc* __restrict__ insts, int ninst, int ntiles, const MLPDevice* __restrict__ mlp, int cur,
           int qout, double abt11) {
  __shared__ MLPShared S;
  mlp_tc_setup(S, *mlp);
  uint32_t phase = 0;
  uint32_t* tile_status = insts[0].status;   // the instance of the CTA's last tile (teardown status)
  C2PTileIn t{}, tn{};
  if ((int)blockIdx.x < ntiles) c2p_load(insts, ninst, blockIdx.x, cur, t);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int next = tile + (int)gridDim.x;
    if (next < ntiles) c2p_load(insts, ninst, next, cur, tn);   // in flight during this tile
    if (next + (int)gridDim.x < ntiles) {                        // the tile after it goes to L2
      int bn = next + (int)gridDim.x;
      const InstDesc& In = tile_inst(insts, ninst, LK_C2P, bn);
      if (In.c2p == 2 && In.c2p_tc) c2p_prefetch(In, bn, cur);
    }
    if (t.use) {
      const InstDesc& I = *t.I;
      tile_status = I.status;
      LearnedOut r;
      if (!learned_point(S, phase, t.in, I.gamma, I.eps1_c2p, I.counters, t.valid, r)) {
        if (threadIdx.x == 0) atomicOr(I.status, ST_TC_TIMEOUT);
        break;   // every thread of the CTA sees the same result
      }
      learned_stats(mlp->stats, t.valid, r.it);
      const uint32_t st = __reduce_or_sync(0xffffffffu, t.valid ? r.st : 0u);
      if (st && (threadIdx.x & 31) == 0) atomicOr(I.status, st);
      if (t.valid) {
        const long long fs = I.fstride, pc = t.pc;
        double* pn = I.prim[1 - cur];
        double pv[NPRIM];
        pv[P_RHO] = r.o.rho; pv[P_P] = r.o.p; pv[P_VX] = r.o.vx; pv[P_VY] = r.o.vy; pv[P_VZ] = r.o.vz;
        pn[P_RHO * fs + pc] = r.o.rho; pn[P_P * fs + pc] = r.o.p;
        pn[P_VX * fs + pc] = r.o.vx; pn[P_VY * fs + pc] = r.o.vy; pn[P_VZ * fs + pc] = r.o.vz;
#pragma unroll
        for (int c = P_PSI; c < NPRIM; ++c) pv[c] = t.fn[c - P_PSI];
        if (!I.primitive_rec) begin_step_point(I, abt11, I.aux[1 - cur], I.stage[qout], pc, pv);
      }
    }
    t = tn;
  }
  mlp_tc_teardown(S, phase, tile_status);
}

// network seeds of n states (SoA 11 x n conserved), tensor-core form
__global__ void __launch_bounds__(TC_ROWS, C2P_CTAS_PER_SM)
k_predict_tc(long long n, const MLPDevice* __restrict__ mlp, const double* __restrict__ cons,
             double* __restrict__ pseed, uint32_t* __restrict__ err_status, uint32_t max_polls, uint32_t self_test) {
  __shared__ MLPShared S;
  mlp_tc_setup(S, *mlp, max_polls, self_test);
  uint32_t phase = 0;
  const long long ntiles = (n + TC_ROWS - 1) / TC_ROWS;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long i0 = tile * TC_ROWS + threadIdx.x;
    const long long i = i0 < n ? i0 : n - 1;
    float f[MLP_IN];
    c2p_features(cons[i], cons[n + i], cons[2 * n + i], cons[3 * n + i], cons[4 * n + i], cons[5 * n + i],
                 cons[6 * n + i], cons[7 * n + i], cons[8 * n + i], cons[9 * n + i], cons[10 * n + i], f);
    float y = 0.0f;
    if (!mlp_tc_tile(S, phase, f, y)) {
      if (threadIdx.x == 0) atomicOr(err_status, ST_TC_TIMEOUT);
      break;
    }
    if (i0 < n) pseed[i] = cons[i] * (double)__expf(y * S.sd_y + S.mu_y);
  }
  mlp_tc_teardown(S, phase, err_status);
}

int c2p_grid(long long ntiles, int ctas_per_sm = C2P_CTAS_PER_SM) {
  const long long g = (long long)ctas_per_sm * 148;
  return (int)(ntiles < g ? (ntiles < 1 ? 1 : ntiles) : g);
}

}  // namespace

int c2p_tiles(int imax, int jmax) {
  return (int)(((long long)(imax + 1) * (jmax + 1) + TC_ROWS - 1) / TC_ROWS);
}

cudaError_t launch_c2p_step(cudaStream_t st, const InstDesc* d, int ninst, int ntiles, const MLPDevice* mlp, int cur,
                            int qout, double abt11) {
  k_c2p_step<<<c2p_grid(ntiles, C2P_STEP_CTAS_PER_SM), TC_ROWS, 0, st>>>(d, ninst, ntiles, mlp, cur, qout, abt11);
  return cudaGetLastError();
}

cudaError_t launch_predict_tc(long long n, const MLPDevice* mlp, const double* cons, double* pseed,
                              uint32_t* err_status, cudaStream_t st, bool self_test) {
  // the self-test bounds its waits tightly: the first one is meant to run out
  k_predict_tc<<<c2p_grid((n + TC_ROWS - 1) / TC_ROWS), TC_ROWS, 0, st>>>(n, mlp, cons, pseed, err_status,
                                                                          self_test ? 64u : TC_MAX_POLLS,
                                                                          self_test ? 1u : 0u);
  return cudaGetLastError();
}

}  // namespace cueva
