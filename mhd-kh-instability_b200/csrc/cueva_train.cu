// cueva_train.cu -- training and batch inference of the learned con2prim
// seed (cueva_mlp.cuh), on the GPU with this file's own kernels:
//   * synthetic (conserved, primitive) pairs from a counter-based generator;
//   * feature extraction and normalisation statistics;
//   * minibatch SGD with Adam: forward and backward passes as small tiled
//     FP32 GEMMs over bf16-rounded weights (the same rounding the inference
//     kernels read), SiLU and its derivative, bias sums, loss;
//   * batch con2prim for the ablation: Cardano, network seed + Newton, or a
//     given seed + Newton, with the Newton iteration count per state.
// The C-ABI entry points are declared in include/cueva.h.
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/cueva.h"
#include "cueva_common.cuh"
#include "cueva_launch.h"
#include "cueva_mlp.cuh"

using namespace cueva;

#define TRY(x)                                                                               \
  do {                                                                                       \
    cudaError_t e_ = (x);                                                                    \
    if (e_ != cudaSuccess) return cueva_fail(CUEVA_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {

// ------------------------------------------------------------ random numbers
// SplitMix64 finaliser (Steele, Lea & Flood 2014) over (seed, index, stream):
// every draw is a pure function of its counter, so the data set does not
// depend on the launch shape.
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double uni(unsigned long long seed, long long i, int k) {
  const unsigned long long h = mix64(seed ^ mix64((unsigned long long)i * 64ull + (unsigned long long)k));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);   // [0, 1)
}
__device__ __forceinline__ double gauss(unsigned long long seed, long long i, int k) {
  const double u1 = 1.0 - uni(seed, i, k), u2 = uni(seed, i, k + 1);   // Box-Muller
  return sqrt(-2.0 * log(u1)) * cos(2.0 * CUDART_PI * u2);
}
__device__ __forceinline__ void unit_vector(unsigned long long seed, long long i, int k, double& x, double& y,
                                            double& z) {
  const double c = 2.0 * uni(seed, i, k) - 1.0, ph = 2.0 * CUDART_PI * uni(seed, i, k + 1);
  const double s = sqrt(fmax(0.0, 1.0 - c * c));
  x = s * cos(ph); y = s * sin(ph); z = c;
}

// synthetic states: rho log-uniform [1e-3, 10], p log-uniform [1e-4, 10],
// W uniform [1, 20], magnetisation |B|^2 / (rho h) log-uniform [1e-3, 10],
// isotropic directions of v and B, E = -v x B + N(0, 1e-3) per component
__global__ void k_synthetic(long long n, unsigned long long seed, double gamma, double* cons, double* prims) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double rho = pow(10.0, -3.0 + 4.0 * uni(seed, i, 0));
    const double p = pow(10.0, -4.0 + 5.0 * uni(seed, i, 1));
    const double W = 1.0 + 19.0 * uni(seed, i, 2);
    const double sig = pow(10.0, -3.0 + 4.0 * uni(seed, i, 3));
    double ux, uy, uz, bx, by, bz;
    unit_vector(seed, i, 4, ux, uy, uz);
    unit_vector(seed, i, 6, bx, by, bz);
    const double vm = sqrt(1.0 - 1.0 / (W * W));
    const double vx = vm * ux, vy = vm * uy, vz = vm * uz;
    const double h = rho + gamma / (gamma - 1.0) * p;
    const double Bm = sqrt(sig * h);
    const double Bx = Bm * bx, By = Bm * by, Bz = Bm * bz;
    const double Ex = -(vy * Bz - vz * By) + 1.0e-3 * gauss(seed, i, 8);
    const double Ey = -(vz * Bx - vx * Bz) + 1.0e-3 * gauss(seed, i, 10);
    const double Ez = -(vx * By - vy * Bx) + 1.0e-3 * gauss(seed, i, 12);
    const Cons c = startconvar(rho, p, vx, vy, vz, Ex, Ey, Ez, Bx, By, Bz, gamma);
    const double cv[11] = {c.D, c.tau, c.Sx, c.Sy, c.Sz, Ex, Ey, Ez, Bx, By, Bz};
#pragma unroll
    for (int f = 0; f < 11; ++f) cons[f * n + i] = cv[f];
    const double pv[5] = {rho, p, vx, vy, vz};
#pragma unroll
    for (int f = 0; f < 5; ++f) prims[f * n + i] = pv[f];
  }
}

// raw features and target log(p/D) of n states
__global__ void k_features(long long n, const double* cons, const double* p, float* X, float* T) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float f[MLP_IN];
    c2p_features(cons[i], cons[n + i], cons[2 * n + i], cons[3 * n + i], cons[4 * n + i], cons[5 * n + i],
                 cons[6 * n + i], cons[7 * n + i], cons[8 * n + i], cons[9 * n + i], cons[10 * n + i], f);
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) X[i * MLP_IN + k] = f[k];
    if (T) T[i] = (float)log(p[i] / cons[i]);
  }
}

// sums and sums of squares of the 7 columns (6 features + target)
__global__ void k_moments(long long n, const float* X, const float* T, double* acc) {
  double s[14] = {};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      const double v = (k < MLP_IN) ? (double)X[i * MLP_IN + k] : (double)T[i];
      s[k] += v; s[7 + k] += v * v;
    }
  }
#pragma unroll
  for (int k = 0; k < 14; ++k) {
    double v = s[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&acc[k], v);
  }
}

// minibatch rows (uniform with replacement; all rows when seed == 0) with
// the normalisation applied
__global__ void k_gather(long long n, int B, unsigned long long seed, long long step, const float* X, const float* T,
                         const float* norm, float* Xb, float* Tb) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const long long row = seed ? (long long)(mix64(seed ^ mix64((unsigned long long)step * 1048576ull + b)) % (unsigned long long)n)
                             : (long long)b;
#pragma unroll
  for (int k = 0; k < MLP_IN; ++k) Xb[b * MLP_IN + k] = (X[row * MLP_IN + k] - norm[k]) / norm[MLP_IN + k];
  Tb[b] = (T[row] - norm[2 * MLP_IN]) / norm[2 * MLP_IN + 1];
}

// C[m][n] (+)= sum_k A(m,k) B(k,n); A(m,k) = TA ? A[k*lda+m] : A[m*lda+k],
// B(k,n) = TB ? B[n*ldb+k] : B[k*ldb+n]; bias[n] added when non-null;
// with SILU the pre-activation goes to Z and silu(Z) to C.
template <bool TA, bool TB, bool SILU>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const float* __restrict__ A, int lda,
                                              const float* __restrict__ Bm, int ldb, const float* __restrict__ bias,
                                              float* __restrict__ C, int ldc, float* __restrict__ Z) {
  __shared__ float sa[16][17], sb[16][17];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m = blockIdx.y * 16 + ty, nn = blockIdx.x * 16 + tx;
  float acc = 0.0f;
  for (int k0 = 0; k0 < K; k0 += 16) {
    {
      const int mm = blockIdx.y * 16 + ty, kk = k0 + tx;
      sa[ty][tx] = (mm < M && kk < K) ? (TA ? A[(long long)kk * lda + mm] : A[(long long)mm * lda + kk]) : 0.0f;
      const int kb = k0 + ty, nb = blockIdx.x * 16 + tx;
      sb[ty][tx] = (kb < K && nb < N) ? (TB ? Bm[(long long)nb * ldb + kb] : Bm[(long long)kb * ldb + nb]) : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 16; ++k) acc = fmaf(sa[ty][k], sb[k][tx], acc);
    __syncthreads();
  }
  if (m < M && nn < N) {
    if (bias) acc += bias[nn];
    if (SILU) {
      Z[(long long)m * ldc + nn] = acc;
      acc = silu(acc);
    }
    C[(long long)m * ldc + nn] = acc;
  }
}

// loss = mean (y - t)^2 over the batch, dY = 2 (y - t) / B
__global__ void k_loss(int B, const float* Y, const float* T, float* dY, float* loss) {
  float s = 0.0f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    const float d = Y[b] - T[b];
    dY[b] = 2.0f * d / (float)B;
    s += d * d;
  }
  __shared__ float red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = red[0] / (float)B;
}

// dZ = dA * silu'(Z)
__global__ void k_silu_back(long long n, const float* dA, const float* Z, float* dZ) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float z = Z[i], s = sigmoid_fast(z);
    dZ[i] = dA[i] * (s * (1.0f + z * (1.0f - s)));
  }
}

// db[n] = sum_b dZ[b][n]
__global__ void k_colsum(int B, int N, const float* dZ, float* db) {
  const int nn = blockIdx.x;
  float s = 0.0f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) s += dZ[(long long)b * N + nn];
  __shared__ float red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[nn] = red[0];
}

// Adam (Kingma & Ba 2015) and the bf16 rounding of the forward copy
__global__ void k_adam(int n, float* w, float* m, float* v, const float* g, float* wr, float lr, float b1, float b2,
                       float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi; v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + 1.0e-8f);
  w[i] = wi;
  wr[i] = __bfloat162float(__float2bfloat16(wi));
}

__global__ void k_round(int n, const float* w, float* wr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) wr[i] = __bfloat162float(__float2bfloat16(w[i]));
}

// batch con2prim: method 1 Cardano, 2 network seed + Newton (Cardano when it
// fails), 3 Newton from seed[i]; iters[i] = Newton iterations (-1 failed,
// 0 for Cardano)
__global__ void k_c2p_batch(long long n, int method, double gamma, double eps1, const MLPDevice* M,
                            const double* cons, const double* prev, const double* seed, double* out, int* iters) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    C2PIn in{cons[i], cons[n + i], cons[2 * n + i], cons[3 * n + i], cons[4 * n + i], cons[5 * n + i],
             cons[6 * n + i], cons[7 * n + i], cons[8 * n + i], cons[9 * n + i], cons[10 * n + i],
             prev[2 * n + i], prev[3 * n + i], prev[4 * n + i], prev[i], prev[n + i]};
    C2POut o{};
    int it = 0;
    if (method == 1) {
      c2p_cardano(in, gamma, eps1, o, nullptr);
    } else {
      // 2: the network's seed; 4: the network's or the previous pressure,
      // whichever leaves the smaller residual; 3: the given seeds
      const double p0 = (method == 2) ? mlp_pressure_seed(*M, in)
                        : (method == 4) ? c2p_best_seed(in, gamma, mlp_pressure_seed(*M, in)) : seed[i];
      it = c2p_newton(in, gamma, p0, o);
      if (it < 0) c2p_cardano(in, gamma, eps1, o, nullptr);
    }
    out[i] = o.rho; out[n + i] = o.p; out[2 * n + i] = o.vx; out[3 * n + i] = o.vy; out[4 * n + i] = o.vz;
    if (iters) iters[i] = it;
  }
}

// network seeds: per thread in FP32 (tensor == 0), or warp-cooperative on
// the tensor cores (tensor == 1; every warp runs full, lanes past n repeat
// state n-1 and store nothing)
__global__ void k_predict(long long n, const MLPDevice* M, const double* cons, double* pseed, int tensor) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long nround = (n + 31) / 32 * 32;
  for (long long i0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; i0 < nround; i0 += stride) {
    const long long i = i0 < n ? i0 : n - 1;
    float f[MLP_IN];
    c2p_features(cons[i], cons[n + i], cons[2 * n + i], cons[3 * n + i], cons[4 * n + i], cons[5 * n + i],
                 cons[6 * n + i], cons[7 * n + i], cons[8 * n + i], cons[9 * n + i], cons[10 * n + i], f);
    const float y = tensor ? mlp_forward_warp(*M, f) : mlp_forward(*M, f);
    if (i0 < n) pseed[i] = cons[i] * (double)__expf(y * M->sd_y + M->mu_y);
  }
}

dim3 grid_for(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return dim3((unsigned)(b < 1 ? 1 : b));
}

}  // namespace

// ---------------------------------------------------------------- the object
struct cueva_mlp {
  int dev = 0;
  int bmax = 0;
  float* w = nullptr;      // FP32 master parameters
  float* wr = nullptr;     // bf16-rounded copy read by the forward passes
  float* m = nullptr;
  float* v = nullptr;
  float* g = nullptr;
  float* norm = nullptr;   // device copy of hnorm
  float hnorm[MLP_NNORM];
  bool normed = false;
  long long step = 0;
  // batch work space
  float *Xb = nullptr, *Tb = nullptr, *Z1 = nullptr, *A1 = nullptr, *Z2 = nullptr, *A2 = nullptr, *Z3 = nullptr,
        *A3 = nullptr, *Y = nullptr, *dY = nullptr, *dA = nullptr, *dZ = nullptr, *loss = nullptr;
  MLPDevice* d_dev = nullptr;
};

namespace {

void free_batch(cueva_mlp* M) {
  for (float** p : {&M->Xb, &M->Tb, &M->Z1, &M->A1, &M->Z2, &M->A2, &M->Z3, &M->A3, &M->Y, &M->dY, &M->dA, &M->dZ})
    if (*p) { cudaFree(*p); *p = nullptr; }
  M->bmax = 0;
}

int32_t ensure_batch(cueva_mlp* M, int B) {
  if (B <= M->bmax) return CUEVA_OK;
  free_batch(M);
  const size_t h = (size_t)B * MLP_H * sizeof(float);
  TRY(cudaMalloc(&M->Xb, (size_t)B * MLP_IN * sizeof(float)));
  TRY(cudaMalloc(&M->Tb, (size_t)B * sizeof(float)));
  for (float** p : {&M->Z1, &M->A1, &M->Z2, &M->A2, &M->Z3, &M->A3, &M->dA, &M->dZ}) TRY(cudaMalloc(p, h));
  TRY(cudaMalloc(&M->Y, (size_t)B * sizeof(float)));
  TRY(cudaMalloc(&M->dY, (size_t)B * sizeof(float)));
  M->bmax = B;
  return CUEVA_OK;
}

template <bool TA, bool TB, bool SILU>
void gemm(int Mr, int N, int K, const float* A, int lda, const float* B, int ldb, const float* bias, float* C,
          int ldc, float* Z = nullptr) {
  const dim3 grid((N + 15) / 16, (Mr + 15) / 16);
  k_gemm<TA, TB, SILU><<<grid, 256>>>(Mr, N, K, A, lda, B, ldb, bias, C, ldc, Z);
}

// forward and backward of one batch already gathered in Xb/Tb; gradients in g
int32_t forward_backward(cueva_mlp* M, int B) {
  const float* W = M->wr;
  float* G = M->g;
  const int H = MLP_H;
  // forward: Z = X W^T + b, A = silu(Z)
  gemm<false, true, true>(B, H, MLP_IN, M->Xb, MLP_IN, W + MLP_OFF_W1, MLP_IN, W + MLP_OFF_B1, M->A1, H, M->Z1);
  gemm<false, true, true>(B, H, H, M->A1, H, W + MLP_OFF_W2, H, W + MLP_OFF_B2, M->A2, H, M->Z2);
  gemm<false, true, true>(B, H, H, M->A2, H, W + MLP_OFF_W3, H, W + MLP_OFF_B3, M->A3, H, M->Z3);
  gemm<false, true, false>(B, 1, H, M->A3, H, W + MLP_OFF_W4, H, W + MLP_OFF_B4, M->Y, 1);
  k_loss<<<1, 256>>>(B, M->Y, M->Tb, M->dY, M->loss);
  // backward
  gemm<true, false, false>(1, H, B, M->dY, 1, M->A3, H, nullptr, G + MLP_OFF_W4, H);         // dW4 = dY^T A3
  k_colsum<<<1, 256>>>(B, 1, M->dY, G + MLP_OFF_B4);
  gemm<false, false, false>(B, H, 1, M->dY, 1, W + MLP_OFF_W4, H, nullptr, M->dA, H);        // dA3 = dY W4
  k_silu_back<<<grid_for((long long)B * H), 256>>>((long long)B * H, M->dA, M->Z3, M->dZ);
  gemm<true, false, false>(H, H, B, M->dZ, H, M->A2, H, nullptr, G + MLP_OFF_W3, H);         // dW3 = dZ3^T A2
  k_colsum<<<H, 256>>>(B, H, M->dZ, G + MLP_OFF_B3);
  gemm<false, false, false>(B, H, H, M->dZ, H, W + MLP_OFF_W3, H, nullptr, M->dA, H);        // dA2 = dZ3 W3
  k_silu_back<<<grid_for((long long)B * H), 256>>>((long long)B * H, M->dA, M->Z2, M->dZ);
  gemm<true, false, false>(H, H, B, M->dZ, H, M->A1, H, nullptr, G + MLP_OFF_W2, H);         // dW2 = dZ2^T A1
  k_colsum<<<H, 256>>>(B, H, M->dZ, G + MLP_OFF_B2);
  gemm<false, false, false>(B, H, H, M->dZ, H, W + MLP_OFF_W2, H, nullptr, M->dA, H);        // dA1 = dZ2 W2
  k_silu_back<<<grid_for((long long)B * H), 256>>>((long long)B * H, M->dA, M->Z1, M->dZ);
  gemm<true, false, false>(H, MLP_IN, B, M->dZ, H, M->Xb, MLP_IN, nullptr, G + MLP_OFF_W1, MLP_IN);  // dW1
  k_colsum<<<H, 256>>>(B, H, M->dZ, G + MLP_OFF_B1);
  TRY(cudaGetLastError());
  return CUEVA_OK;
}

int32_t features_of(long long n, const double* cons, const double* p, float** X, float** T) {
  TRY(cudaMalloc(X, (size_t)n * MLP_IN * sizeof(float)));
  if (T) TRY(cudaMalloc(T, (size_t)n * sizeof(float)));
  k_features<<<grid_for(n), 256>>>(n, cons, p, *X, T ? *T : nullptr);
  TRY(cudaGetLastError());
  return CUEVA_OK;
}

}  // namespace

namespace cueva {
// network as the kernels read it, on the host (for cueva_attach_mlp)
int32_t mlp_device_image(const cueva_mlp* M, MLPDevice* out) {
  if (!M->normed) return cueva_fail(CUEVA_ERR_ARG, "the network has no normalisation (train or set it first)");
  std::vector<float> w(MLP_NPARAM);
  TRY(cudaMemcpy(w.data(), M->w, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
  for (int i = 0; i < MLP_H * MLP_IN; ++i) out->W1[i] = __float2bfloat16(w[MLP_OFF_W1 + i]);
  for (int i = 0; i < MLP_H * MLP_H; ++i) out->W2[i] = __float2bfloat16(w[MLP_OFF_W2 + i]);
  for (int i = 0; i < MLP_H * MLP_H; ++i) out->W3[i] = __float2bfloat16(w[MLP_OFF_W3 + i]);
  for (int i = 0; i < MLP_H; ++i) out->W4[i] = __float2bfloat16(w[MLP_OFF_W4 + i]);
  // biases are FP32 in the kernels; the forward copy rounds them too
  auto rb = [](float x) { return __bfloat162float(__float2bfloat16(x)); };
  for (int i = 0; i < MLP_H; ++i) {
    out->b1[i] = rb(w[MLP_OFF_B1 + i]); out->b2[i] = rb(w[MLP_OFF_B2 + i]); out->b3[i] = rb(w[MLP_OFF_B3 + i]);
  }
  out->b4 = rb(w[MLP_OFF_B4]);
  for (int k = 0; k < MLP_IN; ++k) { out->mu[k] = M->hnorm[k]; out->sd[k] = M->hnorm[MLP_IN + k]; }
  out->mu_y = M->hnorm[2 * MLP_IN];
  out->sd_y = M->hnorm[2 * MLP_IN + 1];
  out->stats = nullptr;
  return CUEVA_OK;
}
int mlp_device_of(const cueva_mlp* M) { return M->dev; }
}  // namespace cueva

namespace {
int32_t refresh_device_image(cueva_mlp* M) {
  MLPDevice h;
  if (int32_t e = mlp_device_image(M, &h)) return e;
  TRY(cudaMemcpy(M->d_dev, &h, sizeof(MLPDevice), cudaMemcpyHostToDevice));
  return CUEVA_OK;
}
}  // namespace

extern "C" {

int32_t cueva_mlp_create(int32_t device, uint64_t seed, cueva_mlp** out) {
  if (!out) return cueva_fail(CUEVA_ERR_ARG, "null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return cueva_fail(CUEVA_ERR_CUDA, "no CUDA device available");
  }
  if (device < 0 || device >= ndev) return cueva_fail(CUEVA_ERR_ARG, "device ordinal out of range");
  TRY(cudaSetDevice(device));
  cueva_mlp* M = new cueva_mlp();
  M->dev = device;
  // He-uniform weights, zero biases (std::mt19937_64: the initial network is
  // a function of the seed only)
  std::vector<float> w(MLP_NPARAM, 0.0f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int off, int fan_out, int fan_in) {
    const double a = std::sqrt(6.0 / fan_in);
    std::uniform_real_distribution<double> U(-a, a);
    for (int i = 0; i < fan_out * fan_in; ++i) w[off + i] = (float)U(rng);
  };
  fill(MLP_OFF_W1, MLP_H, MLP_IN);
  fill(MLP_OFF_W2, MLP_H, MLP_H);
  fill(MLP_OFF_W3, MLP_H, MLP_H);
  fill(MLP_OFF_W4, 1, MLP_H);
  for (int k = 0; k < MLP_NNORM; ++k) M->hnorm[k] = (k >= MLP_IN && k < 2 * MLP_IN) || k == 2 * MLP_IN + 1 ? 1.0f : 0.0f;
  cudaError_t e = cudaSuccess;
  for (float** p : {&M->w, &M->wr, &M->m, &M->v, &M->g})
    if (e == cudaSuccess) e = cudaMalloc(p, MLP_NPARAM * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&M->norm, MLP_NNORM * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&M->loss, sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&M->d_dev, sizeof(MLPDevice));
  if (e == cudaSuccess) e = cudaMemcpy(M->w, w.data(), MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(M->m, 0, MLP_NPARAM * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(M->v, 0, MLP_NPARAM * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(M->norm, M->hnorm, sizeof M->hnorm, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_round<<<(MLP_NPARAM + 255) / 256, 256>>>(MLP_NPARAM, M->w, M->wr);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    cueva_mlp_destroy(M);
    return cueva_fail(CUEVA_ERR_CUDA, std::string("network set-up: ") + cudaGetErrorString(e));
  }
  *out = M;
  return CUEVA_OK;
}

int32_t cueva_mlp_destroy(cueva_mlp* M) {
  if (!M) return CUEVA_OK;
  cudaSetDevice(M->dev);
  cudaDeviceSynchronize();
  free_batch(M);
  for (float* p : {M->w, M->wr, M->m, M->v, M->g, M->norm, M->loss})
    if (p) cudaFree(p);
  if (M->d_dev) cudaFree(M->d_dev);
  delete M;
  return CUEVA_OK;
}

int32_t cueva_mlp_get_params(cueva_mlp* M, float* host, int32_t n) {
  if (!M || !host || n != MLP_NPARAM + MLP_NNORM)
    return cueva_fail(CUEVA_ERR_ARG, "expected " + std::to_string(MLP_NPARAM + MLP_NNORM) + " floats");
  TRY(cudaSetDevice(M->dev));
  TRY(cudaMemcpy(host, M->w, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
  std::memcpy(host + MLP_NPARAM, M->hnorm, sizeof M->hnorm);
  return CUEVA_OK;
}

int32_t cueva_mlp_set_params(cueva_mlp* M, const float* host, int32_t n) {
  if (!M || !host || n != MLP_NPARAM + MLP_NNORM)
    return cueva_fail(CUEVA_ERR_ARG, "expected " + std::to_string(MLP_NPARAM + MLP_NNORM) + " floats");
  TRY(cudaSetDevice(M->dev));
  TRY(cudaMemcpy(M->w, host, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice));
  std::memcpy(M->hnorm, host + MLP_NPARAM, sizeof M->hnorm);
  TRY(cudaMemcpy(M->norm, M->hnorm, sizeof M->hnorm, cudaMemcpyHostToDevice));
  k_round<<<(MLP_NPARAM + 255) / 256, 256>>>(MLP_NPARAM, M->w, M->wr);
  TRY(cudaGetLastError());
  M->normed = true;
  return refresh_device_image(M);
}

int32_t cueva_mlp_synthetic_pairs(int32_t device, int64_t n, uint64_t seed, double gamma, double* d_cons,
                                  double* d_prims, void* stream) {
  if (n <= 0 || !d_cons || !d_prims) return cueva_fail(CUEVA_ERR_ARG, "bad arguments");
  TRY(cudaSetDevice(device));
  k_synthetic<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(n, seed, gamma, d_cons, d_prims);
  TRY(cudaGetLastError());
  return CUEVA_OK;
}

int32_t cueva_mlp_fit_normalisation(cueva_mlp* M, const double* d_cons, const double* d_p, int64_t n) {
  if (!M || n <= 1 || !d_cons || !d_p) return cueva_fail(CUEVA_ERR_ARG, "bad arguments");
  TRY(cudaSetDevice(M->dev));
  float *X = nullptr, *T = nullptr;
  double* acc = nullptr;
  int32_t rc = features_of(n, d_cons, d_p, &X, &T);
  if (!rc) {
    cudaError_t e = cudaMalloc(&acc, 14 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(acc, 0, 14 * sizeof(double));
    if (e == cudaSuccess) {
      k_moments<<<grid_for(n), 256>>>(n, X, T, acc);
      e = cudaGetLastError();
    }
    double h[14];
    if (e == cudaSuccess) e = cudaMemcpy(h, acc, sizeof h, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = cueva_fail(CUEVA_ERR_CUDA, cudaGetErrorString(e));
    else {
      for (int k = 0; k < 7; ++k) {
        const double mu = h[k] / n, var = h[7 + k] / n - mu * mu;
        const double sd = std::sqrt(var > 1e-12 ? var : 1e-12);
        if (k < MLP_IN) { M->hnorm[k] = (float)mu; M->hnorm[MLP_IN + k] = (float)sd; }
        else { M->hnorm[2 * MLP_IN] = (float)mu; M->hnorm[2 * MLP_IN + 1] = (float)sd; }
      }
      M->normed = true;
      e = cudaMemcpy(M->norm, M->hnorm, sizeof M->hnorm, cudaMemcpyHostToDevice);
      if (e != cudaSuccess) rc = cueva_fail(CUEVA_ERR_CUDA, cudaGetErrorString(e));
    }
  }
  if (X) cudaFree(X);
  if (T) cudaFree(T);
  if (acc) cudaFree(acc);
  if (rc) return rc;
  return refresh_device_image(M);
}

int32_t cueva_mlp_train(cueva_mlp* M, const double* d_cons, const double* d_p, int64_t n, int32_t steps,
                        int32_t batch, float lr, uint64_t seed, float* loss_out) {
  if (!M || n <= 0 || steps < 0 || batch <= 0 || !d_cons || !d_p) return cueva_fail(CUEVA_ERR_ARG, "bad arguments");
  if (!M->normed) return cueva_fail(CUEVA_ERR_ARG, "fit the normalisation first");
  TRY(cudaSetDevice(M->dev));
  if (int32_t e = ensure_batch(M, batch)) return e;
  float *X = nullptr, *T = nullptr;
  int32_t rc = features_of(n, d_cons, d_p, &X, &T);
  const float b1 = 0.9f, b2 = 0.999f;
  for (int s = 0; s < steps && !rc; ++s) {
    ++M->step;
    k_gather<<<(batch + 255) / 256, 256>>>(n, batch, seed ? seed : 1ull, M->step, X, T, M->norm, M->Xb, M->Tb);
    rc = forward_backward(M, batch);
    if (rc) break;
    // cosine decay of the learning rate over this call's steps
    const float lr_s = 0.5f * lr * (1.0f + std::cos(3.14159265f * (float)s / (float)(steps > 1 ? steps : 1)));
    const float c1 = 1.0f - std::pow(b1, (float)M->step), c2 = 1.0f - std::pow(b2, (float)M->step);
    k_adam<<<(MLP_NPARAM + 255) / 256, 256>>>(MLP_NPARAM, M->w, M->m, M->v, M->g, M->wr, lr_s, b1, b2, c1, c2);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = cueva_fail(CUEVA_ERR_CUDA, cudaGetErrorString(e));
  }
  if (!rc && loss_out) {
    cudaError_t e = cudaMemcpy(loss_out, M->loss, sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = cueva_fail(CUEVA_ERR_CUDA, cudaGetErrorString(e));
  }
  if (X) cudaFree(X);
  if (T) cudaFree(T);
  if (rc) return rc;
  return refresh_device_image(M);
}

int32_t cueva_mlp_gradients(cueva_mlp* M, const double* d_cons, const double* d_p, int32_t n, float* grads,
                            float* loss_out) {
  if (!M || n <= 0 || !d_cons || !d_p || !grads) return cueva_fail(CUEVA_ERR_ARG, "bad arguments");
  TRY(cudaSetDevice(M->dev));
  if (int32_t e = ensure_batch(M, n)) return e;
  float *X = nullptr, *T = nullptr;
  int32_t rc = features_of(n, d_cons, d_p, &X, &T);
  if (!rc) {
    k_gather<<<(n + 255) / 256, 256>>>(n, n, 0ull, 0, X, T, M->norm, M->Xb, M->Tb);
    rc = forward_backward(M, n);
  }
  if (!rc) {
    cudaError_t e = cudaMemcpy(grads, M->g, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && loss_out) e = cudaMemcpy(loss_out, M->loss, sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = cueva_fail(CUEVA_ERR_CUDA, cudaGetErrorString(e));
  }
  if (X) cudaFree(X);
  if (T) cudaFree(T);
  return rc;
}

int32_t cueva_mlp_predict(cueva_mlp* M, const double* d_cons, int64_t n, double* d_pseed, int32_t tensor_cores) {
  if (!M || n <= 0 || !d_cons || !d_pseed) return cueva_fail(CUEVA_ERR_ARG, "bad arguments");
  if (!M->normed) return cueva_fail(CUEVA_ERR_ARG, "the network has no normalisation");
  TRY(cudaSetDevice(M->dev));
  if (tensor_cores < 0 || tensor_cores > 3) return cueva_fail(CUEVA_ERR_ARG, "tensor_cores must be 0, 1, 2 or 3");
  if (tensor_cores >= 2) {
    // tcgen05 tiles of 128 states; a bounded wait that runs out is reported
    uint32_t* d_err = nullptr;
    TRY(cudaMalloc(&d_err, sizeof(uint32_t)));
    cudaError_t e = cudaMemset(d_err, 0, sizeof(uint32_t));
    if (e == cudaSuccess) e = launch_predict_tc(n, M->d_dev, d_cons, d_pseed, d_err, 0, tensor_cores == 3);
    uint32_t herr = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&herr, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    cudaFree(d_err);
    if (e != cudaSuccess) return cueva_fail(CUEVA_ERR_CUDA, cudaGetErrorString(e));
    if (herr) return cueva_fail(CUEVA_ERR_PHYSICS, "a tensor-core wait ran out (status 64)");
    return CUEVA_OK;
  }
  // whole warps: the grid covers n rounded up to 32 in multiples of the block
  k_predict<<<grid_for((n + 31) / 32 * 32), 256>>>(n, M->d_dev, d_cons, d_pseed, tensor_cores ? 1 : 0);
  TRY(cudaGetLastError());
  TRY(cudaDeviceSynchronize());
  return CUEVA_OK;
}

int32_t cueva_c2p_batch(int32_t device, int32_t method, const cueva_mlp* M, double gamma, double eps1,
                        const double* d_cons, const double* d_prev, const double* d_seed, int64_t n, double* d_out,
                        int32_t* d_iters) {
  if (n <= 0 || !d_cons || !d_prev || !d_out) return cueva_fail(CUEVA_ERR_ARG, "bad arguments");
  if (method < 1 || method > 4)
    return cueva_fail(CUEVA_ERR_ARG, "method must be 1 (Cardano), 2 (network), 3 (seed) or 4 (network or previous p)");
  if ((method == 2 || method == 4) && (!M || !M->normed))
    return cueva_fail(CUEVA_ERR_ARG, "methods 2 and 4 need a trained network");
  if (method == 3 && !d_seed) return cueva_fail(CUEVA_ERR_ARG, "method 3 needs seeds");
  TRY(cudaSetDevice(device));
  k_c2p_batch<<<grid_for(n), 256>>>(n, method, gamma, eps1, (method == 2 || method == 4) ? M->d_dev : nullptr, d_cons, d_prev, d_seed,
                                    d_out, d_iters);
  TRY(cudaGetLastError());
  TRY(cudaDeviceSynchronize());
  return CUEVA_OK;
}

}  // extern "C"
