// cueva_mlp.cuh -- learned con2prim seed (6 -> 64 -> 64 -> 64 -> 1, SiLU).
// Until a trained network is attached the learned path falls back to the
// Cardano solve, which is also its judge.
#pragma once
#include "cueva_point.cuh"

namespace cueva {

__device__ __forceinline__ uint32_t c2p_learned(const C2PIn& in, double gamma, double eps1, const void* mlp,
                                                C2POut& o, unsigned long long* cnt) {
  (void)mlp;
  return c2p_cardano(in, gamma, eps1, o, cnt);
}

}  // namespace cueva
