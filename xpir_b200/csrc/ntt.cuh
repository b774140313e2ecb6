// The reference's lazy DIF NTT (crypto/NFLlib.hpp:450-537) on one polynomial held in
// shared memory, shared by the import and the query encryption (forward twiddles) and the
// client-side decryption (inverse twiddles after a bit-reversal, crypto/NFLlib.hpp:548-566).
// All threads of the block take part.  Its layers: log2(N)-2 radix-2 layers (inputs and
// outputs in [0, 2p)), then the last two layers fused per group of four.
#pragma once

#include <stdint.h>

#include "modarith.cuh"

namespace xpir {

// Position of coefficient idx in a swizzled shared-memory polynomial: the low 4 bits of
// the word index XORed with bits 7..4, so that the passes of ntt_lazy_rb (and the
// callers' coefficient-order loops) read and write shared memory with few or no bank
// conflicts.  Callers of ntt_lazy_rb index their polynomial through swz().
__device__ __forceinline__ uint32_t swz(uint32_t idx) { return idx ^ ((idx >> 4) & 15u); }

// One radix-2 layer of the lazy DIF butterfly on R register-held coefficients whose
// indices are base | (r << lo): the pair differs in bit `lo + RB` of the index, and the
// twiddle index is the lower index modulo the layer's half-length (the twiddles of layer
// `half` start at w + N - 2*half).
template <int R, int RB>
__device__ __forceinline__ void rb_layer(uint64_t (&x)[R], uint32_t base, uint32_t lo, const uint64_t *w,
                                         const uint64_t *ws, uint32_t N, uint64_t p) {
  const uint64_t p2 = p << 1;
  const uint32_t half = 1u << (lo + RB), off = N - 2 * half;
  const uint32_t ib = base & (half - 1);
#pragma unroll
  for (uint32_t r = 0; r < (uint32_t)R; r++) {
    if (r & (1u << RB)) continue;
    const uint32_t i = ib | ((r & ((1u << RB) - 1)) << lo);
    const uint64_t u0 = x[r], u1 = x[r | (1u << RB)];
    uint64_t t0 = u0 + u1;
    t0 = (t0 >= p2) ? t0 - p2 : t0;
    const uint64_t t1 = u0 - u1 + p2;
    x[r] = t0;
    x[r | (1u << RB)] = shoup_lazy(t1, __ldg(w + off + i), __ldg(ws + off + i), p);
  }
}

// Layers RB = LR-1 .. 0 of one pass, skipping those on index bits below `min_bit`.
template <int LR, int RB>
__device__ __forceinline__ void rb_layers(uint64_t (&x)[1 << LR], uint32_t base, uint32_t lo, uint32_t min_bit,
                                          const uint64_t *w, const uint64_t *ws, uint32_t N, uint64_t p) {
  if constexpr (RB >= 0) {
    if (lo + RB >= min_bit) rb_layer<1 << LR, RB>(x, base, lo, w, ws, N, p);
    rb_layers<LR, RB - 1>(x, base, lo, min_bit, w, ws, N, p);
  }
}

// The reference's butterflies with its lazy reductions, so its output bits, evaluated
// register-blocked: each thread holds R = 2^LR
// coefficients whose indices differ in LR consecutive bits and runs up to LR layers on
// them before exchanging through shared memory (an N = 4096 transform makes 3 or 4
// shared-memory round trips instead of 11).  Layers on index bits log2(N)-1 .. LR run in
// passes of LR from the top (a short last group also holds the bits just below it,
// untouched); the last pass holds R consecutive coefficients and runs the layers on bits
// LR-1 .. 2 and the fused last two layers.  The first pass takes its inputs from
// load(idx) (the caller's coefficient idx, in [0, 2p)), so a producer can feed the
// transform without a shared-memory round trip; the output is left in s[swz(idx)].
// 512 <= N <= 8192, LR in {3, 4}; any block size.
template <int LR = 4, class Load>
__device__ inline void ntt_lazy_rb(uint64_t *s, const uint64_t *__restrict__ w, const uint64_t *__restrict__ ws,
                                   uint32_t N, uint32_t log_n, uint64_t p, Load load) {
  constexpr uint32_t R = 1u << LR;
  static_assert(LR == 3 || LR == 4, "register blocks of 8 or 16 coefficients");
  const uint64_t p2 = p << 1;
  const uint32_t groups = N >> LR;
  for (int top = (int)log_n - 1; top >= LR; top -= LR) {
    const uint32_t lo = (uint32_t)top - (LR - 1);
    const bool first = top == (int)log_n - 1;
    if (!first) __syncthreads();
    for (uint32_t g = threadIdx.x; g < groups; g += blockDim.x) {
      const uint32_t base = ((g >> lo) << (lo + LR)) | (g & ((1u << lo) - 1));
      uint64_t x[R];
      if (first) {
#pragma unroll
        for (uint32_t r = 0; r < R; r++) x[r] = load(base | (r << lo));
      } else {
#pragma unroll
        for (uint32_t r = 0; r < R; r++) x[r] = s[swz(base | (r << lo))];
      }
      // index bits lo+LR-1 .. lo; bits below LR are left to the last pass
      rb_layers<LR, LR - 1>(x, base, lo, LR, w, ws, N, p);
#pragma unroll
      for (uint32_t r = 0; r < R; r++) s[swz(base | (r << lo))] = x[r];
    }
  }
  __syncthreads();
  const uint64_t w1 = __ldg(w + N - 4 + 1), w1s = __ldg(ws + N - 4 + 1);
  for (uint32_t g = threadIdx.x; g < groups; g += blockDim.x) {
    const uint32_t base = g << LR;
    uint64_t x[R];
#pragma unroll
    for (uint32_t r = 0; r < R; r++) x[r] = s[swz(base | r)];
    rb_layers<LR, LR - 1>(x, base, 0, 2, w, ws, N, p);
#pragma unroll
    for (uint32_t q = 0; q < R; q += 4) {
      const uint64_t u0 = x[q], u1 = x[q + 1], u2 = x[q + 2], u3 = x[q + 3];
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
      x[q] = z0;
      x[q + 1] = z1;
      x[q + 2] = z2;
      x[q + 3] = z3;
    }
#pragma unroll
    for (uint32_t r = 0; r < R; r++) s[swz(base | r)] = x[r];
  }
  __syncthreads();
}

}  // namespace xpir
