// cueva_mlp_tc.cuh -- the learned con2prim seed network on the sm_100a
// tensor cores (tcgen05): tiles of 128 states, one state per thread of a
// 128-thread CTA.
//
// Per tile: every thread writes its normalised features as one bf16 row of
// the layer-1 A operand in shared memory; thread 0 issues the MMAs of a
// layer (M = 128 states, N = 64 units, K = 16 per instruction) with the
// weights staged once per CTA as the B operand, and commits them to an
// mbarrier; the FP32 accumulator lives in 64 TMEM columns.  Each warp then
// reads its 32 rows (TMEM lanes 32w..32w+31) back with tcgen05.ld, applies
// bias and SiLU, rounds to bf16 and writes the row as the next layer's A
// operand.  The output unit is one more MMA (N = 16, W4 in column 0).
//
// The epilogue is the kernel's arithmetic bottleneck, so it is written for
// the instruction count: with h = (z + b)/2 = fma(z, 1/2, b/2),
//   SiLU(z + b) = (z + b) sigmoid(z + b) = h + h tanh(h),
// one tanh.approx (MUFU) and two FMAs per unit instead of an exponential, a
// reciprocal and their adds.  tanh.approx carries a relative error below
// 2^-10, under the bf16 rounding (2^-9) that every activation gets next, so
// this form and the training form (cueva_mlp.cuh) give seeds that agree to
// the activation rounding; Newton removes the difference.
#pragma once
#include "cueva_mlp.cuh"
#include "cueva_umma.cuh"

namespace cueva {

constexpr int TC_ROWS = 128;             // states per tile = MMA M = threads per CTA
constexpr int TC_NOUT = 16;              // N of the output MMA (column 0 used)
constexpr uint32_t TC_TMEM_COLS = 64;    // FP32 accumulator columns (N)
constexpr uint32_t TC_MAX_POLLS = 1u << 20;   // try_wait suspends for a bounded time per poll

struct __align__(128) MLPShared {
  uint8_t W2[MLP_H * MLP_H * 2];   // B operands (N = 64 outputs x K = 64 inputs), K-major
  uint8_t W3[MLP_H * MLP_H * 2];
  uint8_t A[TC_ROWS * MLP_H * 2];  // hidden activations of the tile (A operand)
  uint8_t W1[MLP_H * 16 * 2];      // K = 6 inputs padded to 16
  uint8_t A1[TC_ROWS * 16 * 2];
  uint8_t W4[TC_NOUT * MLP_H * 2]; // row 0 = output weights, rows 1..15 zero
  float hb1[MLP_H], hb2[MLP_H], hb3[MLP_H];   // biases / 2
  float mu[MLP_IN], isd[MLP_IN];
  float b4, mu_y, sd_y;
  uint64_t bar;                    // MMA completion
  uint32_t taddr;                  // TMEM accumulator
  uint32_t fail;                   // a bounded wait ran out
  uint32_t max_polls;              // bound of every mbarrier wait
  uint32_t self_test;              // 1: issue no MMA, so the first wait runs out (tests the timeout path)
};

__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// The CTA's set-up: network into shared memory (core-matrix layout), the
// mbarrier, and (warp 0) the TMEM columns.  All threads call it.
__device__ __forceinline__ void mlp_tc_setup(MLPShared& S, const MLPDevice& M, uint32_t max_polls = TC_MAX_POLLS,
                                             uint32_t self_test = 0) {
  const int t = threadIdx.x;
  // W2, W3: row n = output unit, 8 consecutive inputs = one 16-byte chunk
  for (int c = t; c < MLP_H * (MLP_H / 8); c += blockDim.x) {
    const int n = c / (MLP_H / 8), kg = c % (MLP_H / 8);
    *reinterpret_cast<uint4*>(S.W2 + umma::kmajor_offset(n, 8 * kg, MLP_H)) =
        *reinterpret_cast<const uint4*>(M.W2 + n * MLP_H + 8 * kg);
    *reinterpret_cast<uint4*>(S.W3 + umma::kmajor_offset(n, 8 * kg, MLP_H)) =
        *reinterpret_cast<const uint4*>(M.W3 + n * MLP_H + 8 * kg);
  }
  for (int e = t; e < MLP_H * 16; e += blockDim.x) {
    const int n = e / 16, k = e % 16;
    *reinterpret_cast<__nv_bfloat16*>(S.W1 + umma::kmajor_offset(n, k, 16)) =
        k < MLP_IN ? M.W1[n * MLP_IN + k] : __float2bfloat16(0.0f);
  }
  for (int e = t; e < TC_NOUT * MLP_H; e += blockDim.x) {
    const int n = e / MLP_H, k = e % MLP_H;
    *reinterpret_cast<__nv_bfloat16*>(S.W4 + umma::kmajor_offset(n, k, MLP_H)) =
        n == 0 ? M.W4[k] : __float2bfloat16(0.0f);
  }
  for (int k = t; k < MLP_H; k += blockDim.x) {
    S.hb1[k] = 0.5f * M.b1[k]; S.hb2[k] = 0.5f * M.b2[k]; S.hb3[k] = 0.5f * M.b3[k];
  }
  if (t < MLP_IN) { S.mu[t] = M.mu[t]; S.isd[t] = 1.0f / M.sd[t]; }
  if (t == 0) {
    S.b4 = M.b4; S.mu_y = M.mu_y; S.sd_y = M.sd_y;
    S.fail = 0;
    S.max_polls = max_polls;
    S.self_test = self_test;
    umma::mbar_init(&S.bar, 1);
    umma::mbar_fence_init();
  }
  if (t < 32) umma::tmem_alloc(&S.taddr, TC_TMEM_COLS);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
}

// Releases the TMEM columns (all threads call it, after their last tile).
// After a timed-out wait the MMAs of that commit may still be in flight: one
// more bounded wait covers them, and if that runs out too, ST_TC_TEARDOWN
// goes to *status (the columns are released regardless, since a CTA must not
// exit holding TMEM).
__device__ __forceinline__ void mlp_tc_teardown(MLPShared& S, uint32_t phase, uint32_t* status) {
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if (S.fail && threadIdx.x == 0 && !umma::mbar_wait(&S.bar, phase, S.max_polls))   // MMAs still in flight
    atomicOr(status, ST_TC_TEARDOWN);
  __syncthreads();
  if (threadIdx.x < 32) umma::tmem_dealloc(S.taddr, TC_TMEM_COLS);
}

// thread 0: the MMAs of one layer (K = 16 * nk, N from idesc) and their commit
__device__ __forceinline__ void mlp_tc_issue(MLPShared& S, const uint8_t* A, const uint8_t* W, int nk,
                                             uint32_t idesc) {
  umma::fence_after_sync();
  if (S.self_test) return;   // nothing will arrive on the barrier
  const uint32_t a0 = umma::smem_u32(A), w0 = umma::smem_u32(W);
  const uint32_t sbo = (uint32_t)nk * 256u;   // K * 16 bytes between 8-row groups
  for (int s = 0; s < nk; ++s)
    umma::mma_bf16(S.taddr, umma::smem_desc(a0 + 256u * s, 128u, sbo), umma::smem_desc(w0 + 256u * s, 128u, sbo),
                   idesc, s > 0 ? 1u : 0u);
  umma::mma_commit(&S.bar);
}

// all threads: waits for the layer's MMAs; false (for every thread) if the
// wait ran out
__device__ __forceinline__ bool mlp_tc_wait(MLPShared& S, uint32_t& phase) {
  if (!umma::mbar_wait(&S.bar, phase, S.max_polls)) atomicOr(&S.fail, 1u);
  __syncthreads();
  umma::fence_after_sync();
  if (S.fail) return false;   // phase keeps the parity of the commit still outstanding
  phase ^= 1u;
  return true;
}

// hidden-layer epilogue of the thread's row: bias, SiLU, bf16, next A operand
__device__ __forceinline__ void mlp_tc_hidden(MLPShared& S, const float* hb) {
  const int r = threadIdx.x;
  const uint32_t lane_base = S.taddr + ((uint32_t)(r & ~31) << 16);
#pragma unroll
  for (int c0 = 0; c0 < MLP_H; c0 += 16) {
    float v[16];
    umma::tmem_ld16(lane_base + c0, v);
    float a[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const float h = fmaf(v[k], 0.5f, hb[c0 + k]);
      a[k] = fmaf(h, tanh_approx(h), h);
    }
    uint32_t p[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) p[k] = pack_bf16x2(a[2 * k], a[2 * k + 1]);
    *reinterpret_cast<uint4*>(S.A + umma::kmajor_offset(r, c0, MLP_H)) = make_uint4(p[0], p[1], p[2], p[3]);
    *reinterpret_cast<uint4*>(S.A + umma::kmajor_offset(r, c0 + 8, MLP_H)) = make_uint4(p[4], p[5], p[6], p[7]);
  }
  umma::fence_before_sync();
  umma::fence_proxy_async();
  __syncthreads();
}

// One tile: f = the thread's raw features (c2p_features); returns the
// normalised network output in y.  All 128 threads call it; false if a
// bounded wait ran out (then y is not set and the CTA must stop).
__device__ __forceinline__ bool mlp_tc_tile(MLPShared& S, uint32_t& phase, const float (&f)[MLP_IN], float& y) {
  const int r = threadIdx.x;
  float x[MLP_IN];
#pragma unroll
  for (int k = 0; k < MLP_IN; ++k) x[k] = (f[k] - S.mu[k]) * S.isd[k];
  *reinterpret_cast<uint4*>(S.A1 + umma::kmajor_offset(r, 0, 16)) =
      make_uint4(pack_bf16x2(x[0], x[1]), pack_bf16x2(x[2], x[3]), pack_bf16x2(x[4], x[5]), 0u);
  *reinterpret_cast<uint4*>(S.A1 + umma::kmajor_offset(r, 8, 16)) = make_uint4(0u, 0u, 0u, 0u);
  umma::fence_proxy_async();
  __syncthreads();
  constexpr uint32_t kHidden = umma::idesc_bf16_f32(TC_ROWS, MLP_H);
  constexpr uint32_t kOut = umma::idesc_bf16_f32(TC_ROWS, TC_NOUT);
  if (r == 0) mlp_tc_issue(S, S.A1, S.W1, 1, kHidden);
  if (!mlp_tc_wait(S, phase)) return false;
  mlp_tc_hidden(S, S.hb1);
  if (r == 0) mlp_tc_issue(S, S.A, S.W2, MLP_H / 16, kHidden);
  if (!mlp_tc_wait(S, phase)) return false;
  mlp_tc_hidden(S, S.hb2);
  if (r == 0) mlp_tc_issue(S, S.A, S.W3, MLP_H / 16, kHidden);
  if (!mlp_tc_wait(S, phase)) return false;
  mlp_tc_hidden(S, S.hb3);
  if (r == 0) mlp_tc_issue(S, S.A, S.W4, MLP_H / 16, kOut);
  if (!mlp_tc_wait(S, phase)) return false;
  y = umma::tmem_ld1(S.taddr + ((uint32_t)(r & ~31) << 16)) + S.b4;
  umma::fence_before_sync();   // TMEM reads complete before the next tile's MMA
  return true;
}

}  // namespace cueva
