// Reply generation for one recursion level: the in-order lazy Shoup multiply-accumulate
// of XPIR (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:511-595 ->
// crypto/NFLLWE.cpp:176-205 -> crypto/NFLlib.hpp:303-321).
//
// Bit-exactness forces every output coefficient to be one sequential chain over the
// slots 0..n_i-1 of its group:  rop += t_q ; rop -= (rop >= p) ? p : 0,  where
// t_q = x_q*y_q - hi(x_q*y'_q)*p (mod 2^64) and y' = floor(y*2^64/p).  The expensive
// part, t_q, does not depend on rop; only the add/compare/subtract is serial.
//
// One CTA owns a W-coefficient slice of one modulus, one group and C consecutive polys
// ("columns") of the level database, and runs a warp-specialised pipeline:
//
//   warp 0      TMA producer: per tile of E slots, one 4-D tiled load of the C DB
//               columns and one of the query's a/b rows into an NS-stage ring
//               (mbarrier expect-tx completion; slots past the real elements come back
//               as zeros from the TMA out-of-bounds fill, which is exactly XPIR's
//               zero-padding element).
//   warps 1..8  compute: the query Shoup factors y' once per (slot, coefficient) from
//               32-bit partial products (modarith.cuh), then the terms t for both
//               ciphertext halves of all C columns into a double-buffered term tile.
//   C warps     chains: one thread per (half, column, coefficient) consumes the term
//               tiles strictly in slot order.
//
// Every mbarrier wait is bounded; a wait that gives up sets the status word and the CTA
// drains its in-flight copies and returns.
//
// Grid: x = group (fastest: CTAs sharing a query slice run together and hit in L2),
//       y = coefficient slice, z = modulus * column blocks + column block.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"
#include "modarith.cuh"
#include "sm100.cuh"

namespace xpir {
namespace {

constexpr int kW = 16;              // coefficients per slice (128-byte TMA rows)
constexpr int kComputeWarps = 8;
constexpr int kComputeThreads = 32 * kComputeWarps;

struct LevelShape {
  uint64_t n_real, P, n_i;
  uint32_t N, m, col_blocks;
};

template <int C, int E, int NS>
struct Smem {
  static constexpr int kX = E * C * kW;     // DB box  [E][C][W]
  static constexpr int kQ = E * 2 * kW;     // query box [E][2][W]
  static constexpr int kT = 2 * C * E * kW;  // terms [half][C][E][W] per buffer
  static constexpr size_t kBytes = (size_t)(NS * (kX + kQ) + 2 * kT) * 8 + (2 * NS + 4) * 8;
};

template <int C, int E, int NS>
__global__ void __launch_bounds__(32 + kComputeThreads + 32 * C, C <= 2 ? 2 : 1)
    reply_tma_kernel(const __grid_constant__ CUtensorMap tm_db, const __grid_constant__ CUtensorMap tm_q,
                     uint64_t *__restrict__ out, const LevelShape sh, const DevModuli dm, int *status) {
  using S = Smem<C, E, NS>;
  extern __shared__ __align__(128) uint64_t sm[];
  uint64_t *xs = sm;                         // [NS][E][C][W]
  uint64_t *qs = xs + NS * S::kX;            // [NS][E][2][W]
  uint64_t *terms = qs + NS * S::kQ;         // [2][2][C][E][W]
  uint64_t *bars = terms + 2 * S::kT;
  uint64_t *full = bars, *empty = bars + NS, *tfull = bars + 2 * NS, *tempty = bars + 2 * NS + 2;

  const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const uint64_t g = blockIdx.x;
  const int k0 = blockIdx.y * kW;
  const uint32_t c = blockIdx.z / sh.col_blocks;
  const uint32_t cp0 = (blockIdx.z - c * sh.col_blocks) * C;
  const uint64_t p = dm.p[c];
  const uint32_t delta = (uint32_t)dm.shoup_delta[c];
  const uint64_t tiles = (sh.n_i + E - 1) / E;

  if (threadIdx.x == 0) {
    // Every consumer thread arrives on the release barriers, so each thread's own
    // shared-memory reads/writes are ordered before its arrive.
    for (int s = 0; s < NS; s++) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, kComputeThreads);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(tfull + b, kComputeThreads);
      mbar_init(tempty + b, 32 * C);
    }
    mbar_fence_init();
  }
  __syncthreads();

  bool ok = true;
  if (warp == 0) {
    // ---- TMA producer ------------------------------------------------------------
    if (lane == 0) {
      tma_prefetch_desc(&tm_db);
      tma_prefetch_desc(&tm_q);
      constexpr uint32_t kTx = (uint32_t)((S::kX + S::kQ) * 8);
      uint64_t t = 0;
      for (; t < tiles; ++t) {
        const int s = (int)(t % NS);
        if (t >= (uint64_t)NS && !mbar_wait(empty + s, (uint32_t)((t / NS - 1) & 1))) {
          ok = false;
          break;
        }
        mbar_arrive_expect_tx(full + s, kTx);
        const int slot = (int)(t * E);
        tma_load_4d(xs + s * S::kX, &tm_db, k0, (int)c, (int)cp0, (int)(g * sh.n_i) + slot, full + s);
        tma_load_4d(qs + s * S::kQ, &tm_q, k0, (int)c, 0, slot, full + s);
      }
      // Drain: every issued copy must have landed before the CTA exits.
      const uint64_t first = t > (uint64_t)NS ? t - NS : 0;
      for (uint64_t u = first; u < t; ++u) mbar_wait(full + (u % NS), (uint32_t)((u / NS) & 1));
    }
  } else if (warp <= kComputeWarps) {
    // ---- compute warps: query Shoup factors and terms -------------------------------
    const int ct = threadIdx.x - 32;
    for (uint64_t t = 0; t < tiles && ok; ++t) {
      const int s = (int)(t % NS), b = (int)(t & 1);
      if (!mbar_wait(full + s, (uint32_t)((t / NS) & 1))) ok = false;
      if (ok && t >= 2 && !mbar_wait(tempty + b, (uint32_t)((t / 2 - 1) & 1))) ok = false;
      if (!ok) break;
      const uint64_t *xst = xs + s * S::kX;
      const uint64_t *qst = qs + s * S::kQ;
      uint64_t *tb = terms + b * S::kT;
#pragma unroll
      for (int r = 0; r < (E * kW) / kComputeThreads; r++) {
        const int item = ct + r * kComputeThreads;
        const int e = item / kW, k = item % kW;
        const uint64_t ya = qst[(e * 2 + 0) * kW + k];
        const uint64_t yb = qst[(e * 2 + 1) * kW + k];
        const uint64_t ysa = shoup_factor8(ya, p, delta);
        const uint64_t ysb = shoup_factor8(yb, p, delta);
#pragma unroll
        for (int col = 0; col < C; col++) {
          const uint64_t x = xst[(e * C + col) * kW + k];
          tb[((0 * C + col) * E + e) * kW + k] = shoup_lazy(x, ya, ysa, p);
          tb[((1 * C + col) * E + e) * kW + k] = shoup_lazy(x, yb, ysb, p);
        }
      }
      mbar_arrive(empty + s);
      mbar_arrive(tfull + b);
    }
  } else {
    // ---- chain warps: strictly in-order accumulation ---------------------------------
    const int u = threadIdx.x - 32 - kComputeThreads;  // (half, column, coefficient)
    const int h = u / (C * kW), col = (u / kW) % C, k = u % kW;
    uint64_t rop = 0;
    for (uint64_t t = 0; t < tiles; ++t) {
      const int b = (int)(t & 1);
      if (!mbar_wait(tfull + b, (uint32_t)((t / 2) & 1))) {
        ok = false;
        break;
      }
      const uint64_t *tb = terms + b * S::kT + ((h * C + col) * E) * kW + k;
      const uint64_t left = sh.n_i - t * E;
      if (left >= (uint64_t)E) {
        // Loads are issued a batch ahead of the dependent add/compare/subtract so that
        // only the 64-bit chain arithmetic is on the critical path.
        constexpr int kB = 8;
        uint64_t cur[kB], nxt[kB];
#pragma unroll
        for (int j = 0; j < kB; j++) cur[j] = tb[j * kW];
#pragma unroll
        for (int e0 = 0; e0 < E; e0 += kB) {
          if (e0 + kB < E) {
#pragma unroll
            for (int j = 0; j < kB; j++) nxt[j] = tb[(e0 + kB + j) * kW];
          }
#pragma unroll
          for (int j = 0; j < kB; j++) {
            const uint64_t w = rop + cur[j];
            rop = w >= p ? w - p : w;
          }
#pragma unroll
          for (int j = 0; j < kB; j++) cur[j] = nxt[j];
        }
      } else {
        for (int e = 0; e < (int)left; e++) {
          const uint64_t w = rop + tb[e * kW];
          rop = w >= p ? w - p : w;
        }
      }
      mbar_arrive(tempty + b);
    }
    const uint64_t cp = cp0 + col;
    if (ok && cp < sh.P) {
      const uint64_t mN = (uint64_t)sh.m * sh.N;
      out[((g * sh.P + cp) * 2 + h) * mN + (uint64_t)c * sh.N + k0 + k] = rop;
    }
  }
  if (!ok) {
    *(volatile int *)status = kStatusWaitTimeout;
    __threadfence_system();
  }
}

template <int C, int E, int NS>
cudaError_t launch_c(const ReplyLevelArgs &a, const ParamSet &ps, const DevModuli &dm, uint64_t groups,
                     cudaStream_t stream, int *status) {
  // DB level viewed as [element][poly][modulus][coefficient]; query as [slot][half][modulus][coefficient].
  const uint64_t N = ps.N, m = ps.m;
  CUtensorMap tm_db, tm_q;
  const uint64_t db_dims[4] = {N, m, a.P, a.n_real};
  const uint64_t db_strides[3] = {N * 8, m * N * 8, a.P * m * N * 8};
  const uint32_t db_box[4] = {(uint32_t)kW, 1, (uint32_t)C, (uint32_t)E};
  const uint64_t q_dims[4] = {N, m, 2, a.n_i};
  const uint64_t q_strides[3] = {N * 8, m * N * 8, 2 * m * N * 8};
  const uint32_t q_box[4] = {(uint32_t)kW, 1, 2, (uint32_t)E};
  if (!encode_tensor_map_u64_4d(&tm_db, a.db, db_dims, db_strides, db_box) ||
      !encode_tensor_map_u64_4d(&tm_q, a.query, q_dims, q_strides, q_box))
    return cudaErrorInvalidValue;
  using S = Smem<C, E, NS>;
  auto kern = reply_tma_kernel<C, E, NS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::kBytes);
  if (e != cudaSuccess) return e;
  const uint32_t col_blocks = (uint32_t)((a.P + C - 1) / C);
  LevelShape sh{a.n_real, a.P, a.n_i, ps.N, ps.m, col_blocks};
  if (groups > 0x7fffffffull || (uint64_t)m * col_blocks > 65535) return cudaErrorInvalidValue;
  dim3 grid((unsigned)groups, ps.N / kW, (unsigned)(m * col_blocks));
  kern<<<grid, 32 + kComputeThreads + 32 * C, S::kBytes, stream>>>(tm_db, tm_q, a.out, sh, dm, status);
  return cudaGetLastError();
}

}  // namespace

bool reply_level_supported(const ParamSet &ps, uint64_t n_real, uint64_t n_i, uint64_t groups) {
  for (uint32_t c = 0; c < ps.m; c++)
    if (!shoup_factor8_ok(ps.mod[c].p)) return false;
  // TMA coordinates are 32-bit signed.
  return ps.N % kW == 0 && n_real < (1ull << 31) && groups * n_i + 256 < (1ull << 31);
}

cudaError_t launch_reply_level(const ReplyLevelArgs &a, const ParamSet &ps, const DevModuli &dm,
                               cudaStream_t stream, uint32_t *launches, int *status) {
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
  if (!reply_level_supported(ps, a.n_real, a.n_i, active)) return cudaErrorNotSupported;
  if (launches) (*launches)++;
  switch (a.P) {
    case 1: return launch_c<1, 32, 4>(a, ps, dm, active, stream, status);
    case 2: return launch_c<2, 32, 3>(a, ps, dm, active, stream, status);
    case 3: return launch_c<3, 16, 4>(a, ps, dm, active, stream, status);
    case 4: return launch_c<4, 16, 3>(a, ps, dm, active, stream, status);
    case 5: return launch_c<5, 16, 3>(a, ps, dm, active, stream, status);
    case 6: return launch_c<6, 16, 3>(a, ps, dm, active, stream, status);
    case 7: return launch_c<7, 16, 3>(a, ps, dm, active, stream, status);
    default: return launch_c<8, 16, 3>(a, ps, dm, active, stream, status);
  }
}

}  // namespace xpir
