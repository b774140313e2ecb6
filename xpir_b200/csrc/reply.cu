// Reply generation for one recursion level: the in-order lazy Shoup multiply-accumulate
// of XPIR (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:511-595 ->
// crypto/NFLLWE.cpp:176-205 -> crypto/NFLlib.hpp:303-321).
//
// Bit-exactness forces every output coefficient to be one sequential chain over the
// slots 0..n_i-1 of its group:  rop += t_q ; rop -= (rop >= p) ? p : 0,  where
// t_q = x_q*y_q - hi(x_q*y'_q)*p (mod 2^64) and y' = floor(y*2^64/p).  The expensive
// part, t_q, has no dependence on rop; only the add/compare/subtract is serial.  So each
// CTA owns a W-coefficient slice of one (group, poly, modulus) and splits its warps:
//
//   * 8 compute warps stream DB and query tiles (E slots x W coefficients) from HBM into
//     an NS-stage shared-memory ring with cp.async, compute the query Shoup factors on
//     the fly (no 128/64 division, see modarith.cuh) and the terms t_q for both
//     ciphertext halves, and write them to a double-buffered term tile;
//   * 2 chain warps (one thread per chain: 2 halves x W coefficients) consume the
//     previous term tile strictly in slot order.
//
// Grid: x = group (fastest, so the CTAs that share a query slice run together and hit
// in L2), y = coefficient slice, z = modulus * P + poly.
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"
#include "modarith.cuh"

namespace xpir {
namespace {

constexpr int kComputeThreads = 256;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = pred ? 16 : 0;  // src-size 0 zero-fills the 16 bytes
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

struct LevelShape {
  uint64_t n_real, P, n_i;
  uint32_t N, m;
};

template <int W, int E, int NS>
__global__ void __launch_bounds__(kComputeThreads + 2 * W)
    reply_level_kernel(const uint64_t *__restrict__ db, const uint64_t *__restrict__ query,
                       uint64_t *__restrict__ out, const LevelShape sh, const DevModuli dm) {
  extern __shared__ __align__(16) uint64_t sm[];
  constexpr int kStageWords = E * 3 * W;  // per slot: x[W], ya[W], yb[W]
  uint64_t *stage = sm;
  uint64_t *terms = sm + NS * kStageWords;  // [2 buffers][2 halves][E][W]

  const uint64_t g = blockIdx.x;
  const uint32_t k0 = blockIdx.y * W;
  const uint32_t c = blockIdx.z / (uint32_t)sh.P;
  const uint64_t cp = blockIdx.z - (uint64_t)c * sh.P;
  const uint64_t p = dm.p[c], sk = dm.shoup_k[c], sd = dm.shoup_delta[c];
  const uint64_t N = sh.N, mN = (uint64_t)sh.m * N;
  const uint64_t tiles = (sh.n_i + E - 1) / E;
  const bool chain = threadIdx.x >= kComputeThreads;

  auto issue = [&](uint64_t tile) {
    uint64_t *st = stage + (tile % NS) * kStageWords;
    constexpr int kChunks = W / 2;  // 16-byte chunks per row
    static_assert((E * 3 * kChunks) % kComputeThreads == 0, "tile copy must split evenly");
#pragma unroll
    for (int r = 0; r < (E * 3 * kChunks) / kComputeThreads; r++) {
      const int q = threadIdx.x + r * kComputeThreads;
      const int row = q / (3 * kChunks);
      const int rem = q - row * 3 * kChunks;
      const int which = rem / kChunks;  // 0: DB word x, 1: query a, 2: query b
      const int ch = rem - which * kChunks;
      const uint64_t slot = tile * E + row;
      const uint64_t *src = query;
      bool ok = slot < sh.n_i;
      if (which == 0) {
        const uint64_t elem = g * sh.n_i + slot;
        ok = ok && elem < sh.n_real;
        if (ok) src = db + (elem * sh.P + cp) * mN + c * N + k0 + 2 * ch;
      } else if (ok) {
        src = query + (slot * 2 + (which - 1)) * mN + c * N + k0 + 2 * ch;
      }
      cp_async16(st + (row * 3 + which) * W + 2 * ch, src, ok);
    }
  };

  if (!chain) {
#pragma unroll
    for (int s = 0; s < NS - 1; s++) {
      if ((uint64_t)s < tiles) issue(s);
      cp_async_commit();
    }
  }

  const int u = threadIdx.x - kComputeThreads;  // chain thread: half u / W, coefficient u % W
  uint64_t rop = 0;
  for (uint64_t it = 0; it <= tiles; ++it) {
    if (!chain) cp_async_wait<NS - 2>();
    __syncthreads();
    if (!chain) {
      if (it + NS - 1 < tiles) issue(it + NS - 1);
      cp_async_commit();
      if (it < tiles) {
        const uint64_t *st = stage + (it % NS) * kStageWords;
        uint64_t *tb = terms + (it & 1) * (2 * E * W);
        static_assert((E * W) % kComputeThreads == 0, "term tile must split evenly");
#pragma unroll
        for (int r = 0; r < (E * W) / kComputeThreads; r++) {
          const int q = threadIdx.x + r * kComputeThreads;
          const int e = q / W, k = q - e * W;
          const uint64_t x = st[(e * 3) * W + k];
          const uint64_t ya = st[(e * 3 + 1) * W + k];
          const uint64_t yb = st[(e * 3 + 2) * W + k];
          tb[e * W + k] = shoup_lazy(x, ya, shoup_factor(ya, p, sk, sd), p);
          tb[E * W + e * W + k] = shoup_lazy(x, yb, shoup_factor(yb, p, sk, sd), p);
        }
      }
    } else if (it >= 1) {
      const uint64_t tile = it - 1;
      const uint64_t *tb = terms + (tile & 1) * (2 * E * W) + (u / W) * (E * W) + (u % W);
      const uint64_t left = sh.n_i - tile * E;
      if (left >= (uint64_t)E) {
#pragma unroll
        for (int e = 0; e < E; e++) {
          rop += tb[e * W];
          rop = rop >= p ? rop - p : rop;
        }
      } else {
        for (int e = 0; e < (int)left; e++) {
          rop += tb[e * W];
          rop = rop >= p ? rop - p : rop;
        }
      }
    }
  }
  if (chain) {
    const uint32_t h = u / W, k = u % W;
    out[((g * sh.P + cp) * 2 + h) * mN + c * N + k0 + k] = rop;
  }
}

template <int W, int E, int NS>
cudaError_t launch_tiled(const ReplyLevelArgs &a, const ParamSet &ps, const DevModuli &dm, uint64_t groups,
                         cudaStream_t stream) {
  const size_t smem = (size_t)(NS * E * 3 * W + 2 * 2 * E * W) * sizeof(uint64_t);
  auto kern = reply_level_kernel<W, E, NS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  LevelShape sh{a.n_real, a.P, a.n_i, ps.N, ps.m};
  if (groups > 0x7fffffffull || ps.N / W > 65535 || ps.m * a.P > 65535) return cudaErrorInvalidValue;
  dim3 grid((unsigned)groups, ps.N / W, (unsigned)(ps.m * a.P));
  kern<<<grid, kComputeThreads + 2 * W, smem, stream>>>(a.db, a.query, a.out, sh, dm);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_reply_level(const ReplyLevelArgs &a, const ParamSet &ps, const DevModuli &dm,
                               cudaStream_t stream, uint32_t *launches) {
  const uint64_t ct_words = 2ull * ps.m * ps.N;
  // Groups whose every slot is past the real elements accumulate only zero terms from
  // a zero start: their replies are exactly zero.  Only groups with data are launched.
  uint64_t active = a.n_i == 0 ? 0 : (a.n_real + a.n_i - 1) / a.n_i;
  if (active > a.n_groups) active = a.n_groups;
  if (active < a.n_groups) {
    cudaError_t e = cudaMemsetAsync(a.out + active * a.P * ct_words, 0,
                                    (a.n_groups - active) * a.P * ct_words * sizeof(uint64_t), stream);
    if (e != cudaSuccess) return e;
  }
  if (active == 0) return cudaSuccess;
  if (launches) (*launches)++;
  return launch_tiled<32, 32, 4>(a, ps, dm, active, stream);
}

}  // namespace xpir
