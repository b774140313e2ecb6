// The reference's lazy DIF NTT on one polynomial held in shared memory, shared by the
// import (forward twiddles) and the client-side decryption (inverse twiddles after a
// bit-reversal, crypto/NFLlib.hpp:548-566).  All threads of the block take part.
#pragma once

#include <stdint.h>

#include "modarith.cuh"

namespace xpir {

// Twiddle layers of the reference NTT: log2(N)-2 radix-2 layers (inputs/outputs in [0,2p)),
// then the last two layers fused per group of four (crypto/NFLlib.hpp:470-535).
__device__ inline void ntt_lazy_smem(uint64_t *s, const uint64_t *__restrict__ w, const uint64_t *__restrict__ ws,
                              uint32_t N, uint32_t log_n, uint64_t p) {
  const uint64_t p2 = p << 1;
  uint32_t half = N >> 1;
  for (uint32_t l = 0; l + 2 < log_n; ++l) {
    __syncthreads();
    const uint32_t lh = log_n - 1 - l;  // log2(half)
    for (uint32_t t = threadIdx.x; t < (N >> 1); t += blockDim.x) {
      const uint32_t i = t & (half - 1);
      const uint32_t idx = ((t >> lh) << (lh + 1)) + i;
      const uint64_t u0 = s[idx], u1 = s[idx + half];
      uint64_t t0 = u0 + u1;
      t0 = (t0 >= p2) ? t0 - p2 : t0;
      const uint64_t t1 = u0 - u1 + p2;
      s[idx] = t0;
      s[idx + half] = shoup_lazy(t1, __ldg(w + i), __ldg(ws + i), p);
    }
    w += half;
    ws += half;
    half >>= 1;
  }
  __syncthreads();
  const uint64_t w1 = __ldg(w + 1), w1s = __ldg(ws + 1);
  for (uint32_t g = threadIdx.x; g < (N >> 2); g += blockDim.x) {
    uint64_t *y = s + 4 * g;
    const uint64_t u0 = y[0], u1 = y[1], u2 = y[2], u3 = y[3];
    uint64_t v0 = u0 + u2;
    v0 = (v0 >= p2) ? v0 - p2 : v0;
    uint64_t v2 = u0 - u2;
    v2 = ((int64_t)v2 < 0) ? v2 + p2 : v2;
    uint64_t v1 = u1 + u3;
    v1 = (v1 >= p2) ? v1 - p2 : v1;
    const uint64_t v3 = shoup_lazy(u1 - u3 + p2, w1, w1s, p);
    uint64_t z0 = v0 + v1;
    z0 = (z0 >= p2) ? z0 - p2 : z0;
    uint64_t z1 = v0 - v1;
    z1 = ((int64_t)z1 < 0) ? z1 + p2 : z1;
    uint64_t z2 = v2 + v3;
    z2 = (z2 >= p2) ? z2 - p2 : z2;
    uint64_t z3 = v2 - v3;
    z3 = ((int64_t)z3 < 0) ? z3 + p2 : z3;
    y[0] = z0;
    y[1] = z1;
    y[2] = z2;
    y[3] = z3;
  }
  __syncthreads();
}

}  // namespace xpir
