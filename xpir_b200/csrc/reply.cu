// Reply generation for one recursion level: the in-order lazy Shoup multiply-accumulate
// of XPIR (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:511-595 ->
// crypto/NFLLWE.cpp:176-205 -> crypto/NFLlib.hpp:303-321).
//
// Bit-exactness forces every output coefficient to be one sequential chain over the
// slots 0..n_i-1 of its group:  rop += t_q ; rop -= (rop >= p) ? p : 0,  where
// t_q = x_q*y_q - hi(x_q*y'_q)*p (mod 2^64) and y' = floor(y*2^64/p).  The expensive
// part, t_q, does not depend on rop; only the add/compare/subtract is serial.
//
// One CTA owns a W-coefficient slice of one modulus and C "columns" of the level
// database -- C consecutive polys of one group's elements, or (group-column tiles, for
// one-poly levels) the poly of C consecutive groups -- and runs a warp-specialised
// pipeline:
//
//   warp 0      TMA producer: per tile of E slots, one 4-D tiled load of the C DB
//               columns (one per group for group columns) and one of the query's a/b
//               rows into an NS-stage ring
//               (mbarrier expect-tx completion; slots past the real elements come back
//               as zeros from the TMA out-of-bounds fill, which is exactly XPIR's
//               zero-padding element).
//   compute     E*W/(2*IPT) threads, IPT slot pairs each: the query Shoup factors y'
//               once per (slot, coefficient) from 32-bit partial products
//               (modarith.cuh), then the terms t for both ciphertext halves of all C
//               columns into a double-buffered term tile.
//   chains      one thread per (half, column, coefficient) consumes the term tiles
//               strictly in slot order.
//
// Every mbarrier wait is bounded; a wait that gives up sets the status word and the CTA
// drains its in-flight copies and returns.
//
// Grid: x = group, or block of C groups (fastest: CTAs sharing a query slice run
//       together and hit in L2), y = coefficient slice, z = modulus * column blocks +
//       column block.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <algorithm>

#include "kernels.h"
#include "modarith.cuh"
#include "sm100.cuh"

namespace xpir {
namespace {

// Tile configuration: W coefficients per slice, C columns, E slots per tile, NS
// pipeline stages, TB term buffers, IPT slot pairs per compute thread and tile.  The C
// columns are C consecutive polys of one element, or with GRP (one-poly levels) the same
// poly of C consecutive groups, which then share every query tile and the Shoup factors
// derived from it.  One chain thread per (half, column, coefficient).
template <int W, int C, int E, int NS, int TB = 2, int IPT = 1, bool GRP = false>
struct Cfg {
  static constexpr int kComputeWarps = E * W / 2 / 32 / IPT;
  static constexpr int kComputeThreads = 32 * kComputeWarps;
  static constexpr int kChainThreads = 2 * C * W;
  static constexpr int kChainWarps = (kChainThreads + 31) / 32;
  static constexpr int kThreads = 32 * (1 + kComputeWarps + kChainWarps);
  // TMA rows start on a 32-byte sector: a slice whose start is only 16-byte aligned
  // (W = 2 mod 4) loads a box two coefficients wider, from the sector boundary below it.
  static constexpr int kBW = (W % 4 == 0) ? W : W + 2;
  static constexpr int kX = E * C * kBW;   // DB box    [E][C][kBW], with GRP [C][E][kBW]
  static constexpr int kQ = E * 2 * kBW;   // query box [E][2][kBW]
  static constexpr int kT = 2 * C * E * W;  // terms     [half][C][E/2][W][2] per buffer
  static constexpr size_t kBytes = (size_t)(NS * (kX + kQ) + TB * kT) * 8 + (2 * NS + 2 * TB) * 8;
  static_assert((TB & (TB - 1)) == 0, "term buffers: a power of two");
  static_assert(E % 2 == 0 && (E * W / 2) % (32 * IPT) == 0, "slot pairs must fill whole warps");
  static_assert(W % 2 == 0, "TMA rows must be multiples of 16 bytes");
  static_assert(!GRP || C > 1, "group columns: at least two groups");
};

// 16-byte shared-memory load/store of two consecutive words.  volatile keeps a batch of
// loads where it is written, ahead of the arithmetic that consumes the previous batch.
__device__ __forceinline__ void lds_v2(const uint64_t *p, uint64_t &a, uint64_t &b) {
  asm volatile("ld.shared.v2.u64 {%0, %1}, [%2];\n" : "=l"(a), "=l"(b) : "r"(smem_addr(p)) : "memory");
}
__device__ __forceinline__ void sts_v2(uint64_t *p, uint64_t a, uint64_t b) {
  asm volatile("st.shared.v2.u64 [%0], {%1, %2};\n" ::"r"(smem_addr(p)), "l"(a), "l"(b) : "memory");
}
// The same store as plain C++, which the compiler may schedule freely (the mbarrier
// arrive that publishes the tile orders it).
__device__ __forceinline__ void st_v2(uint64_t *p, uint64_t a, uint64_t b) {
  *reinterpret_cast<ulonglong2 *>(p) = make_ulonglong2(a, b);
}

struct LevelShape {
  uint64_t n_real, P, n_i;
  uint32_t N, m, col_blocks;
  uint64_t groups;  // groups with data (GRP tiles write only these)
  WaitTest wait_test;
};


// The work of one CTA: group g, coefficient slice blockIdx.y, modulus / column block
// blockIdx.z, with the DB and query tensor maps and the output of its task.  The last
// slice may extend past N (W need not divide N): the TMA fills those coefficients with
// zeros and their chains write nothing.
template <int W, int C, int E, int NS, int TB, int IPT, bool GRP>
__device__ __forceinline__ void reply_tile(const CUtensorMap *tm_db, const CUtensorMap *tm_q,
                                           uint64_t *__restrict__ out, const uint64_t g,
                                           const LevelShape &sh, const DevModuli &dm, int *status) {
  using S = Cfg<W, C, E, NS, TB, IPT, GRP>;
  constexpr int kComputeWarps = S::kComputeWarps;
  constexpr int kComputeThreads = S::kComputeThreads;
  constexpr int kW = W;
  extern __shared__ __align__(128) uint64_t sm[];
  uint64_t *xs = sm;                         // [NS][E][C][W]
  uint64_t *qs = xs + NS * S::kX;            // [NS][E][2][W]
  uint64_t *terms = qs + NS * S::kQ;         // [TB][2][C][E/2][W][2]
  uint64_t *bars = terms + TB * S::kT;
  uint64_t *full = bars, *empty = bars + NS, *tfull = bars + 2 * NS, *tempty = bars + 2 * NS + TB;

  const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int k0 = blockIdx.y * kW;
  const int ka = k0 & ~3, off = k0 - ka;  // sector-aligned box start; the slice begins at off
  const uint32_t c = blockIdx.z / sh.col_blocks;
  const uint32_t cp0 = (blockIdx.z - c * sh.col_blocks) * C;
  const uint64_t p = dm.p[c];
  const uint32_t delta = (uint32_t)dm.shoup_delta[c];
  const uint64_t np = opaque(0 - p);
  const uint32_t tiles = (uint32_t)((sh.n_i + E - 1) / E);
  const uint32_t lim = sh.wait_test.spin_limit ? sh.wait_test.spin_limit : kSpinLimit;

  if (threadIdx.x == 0) {
    // Every consumer thread arrives on the release barriers, so each thread's own
    // shared-memory reads/writes are ordered before its arrive.
    for (int s = 0; s < NS; s++) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, kComputeThreads);
    }
    for (int b = 0; b < TB; b++) {
      mbar_init(tfull + b, kComputeThreads);
      mbar_init(tempty + b, S::kChainThreads);
    }
    mbar_fence_init();
  }
  __syncthreads();

  bool ok = true;
  if (warp == 0) {
    // ---- TMA producer ------------------------------------------------------------
    if (lane == 0) {
      tma_prefetch_desc(tm_db);
      tma_prefetch_desc(tm_q);
      constexpr uint32_t kTx = (uint32_t)((S::kX + S::kQ) * 8);
      uint32_t t = 0;
      for (; t < tiles; ++t) {
        const int s = (int)(t % NS);
        if ((int32_t)t == sh.wait_test.withhold_tile) break;  // test support: starve the consumers
        if (t >= (uint32_t)NS && !mbar_wait(empty + s, (t / NS - 1) & 1, lim)) {
          ok = false;
          break;
        }
        mbar_arrive_expect_tx(full + s, kTx);
        const int slot = (int)t * E;
        if constexpr (GRP) {
#pragma unroll
          for (int col = 0; col < C; col++)
            tma_load_4d(xs + s * S::kX + col * E * S::kBW, tm_db, ka, (int)c, 0,
                        (int)((g * C + col) * sh.n_i) + slot, full + s);
        } else {
          tma_load_4d(xs + s * S::kX, tm_db, ka, (int)c, (int)cp0, (int)(g * sh.n_i) + slot, full + s);
        }
        tma_load_4d(qs + s * S::kQ, tm_q, ka, (int)c, 0, slot, full + s);
      }
      // Drain: every issued copy must have landed before the CTA exits.
      const uint32_t first = t > (uint32_t)NS ? t - NS : 0;
      for (uint32_t u = first; u < t; ++u) mbar_wait(full + (u % NS), (u / NS) & 1);
    }
  } else if (warp <= kComputeWarps) {
    // ---- compute warps: query Shoup factors and terms -------------------------------
    const int ct = threadIdx.x - 32;
    for (uint32_t t = 0; t < tiles && ok; ++t) {
      const int s = (int)(t % NS), b = (int)(t % TB);
      if (!mbar_wait(full + s, (t / NS) & 1, lim)) ok = false;
      if (ok && t >= (uint32_t)TB && !mbar_wait(tempty + b, (t / TB - 1) & 1, lim)) ok = false;
      if (!ok) break;
      const uint64_t *xst = xs + s * S::kX + off;
      const uint64_t *qst = qs + s * S::kQ + off;
      uint64_t *tb = terms + b * S::kT;
      // Thread -> IPT items (coefficient k, slot pair e, e+1); the pair is stored as one
      // 16-byte word so that a chain thread reads two consecutive slots with one load.
      // Several columns: all inputs are loaded before the arithmetic, so the loads of
      // later columns overlap the products of earlier ones (faster for C > 1 on B200;
      // for one column the interleaved form below is slightly faster).
      if constexpr (C > 1) {
#pragma unroll
        for (int it = 0; it < IPT; it++) {
          const int item = ct + it * kComputeThreads;
          const int k = item % kW, ep = item / kW, e = 2 * ep;
          uint64_t x[C][2];
          const uint64_t ya0 = qst[(e * 2 + 0) * S::kBW + k], yb0 = qst[(e * 2 + 1) * S::kBW + k];
          const uint64_t ya1 = qst[(e * 2 + 2) * S::kBW + k], yb1 = qst[(e * 2 + 3) * S::kBW + k];
#pragma unroll
          for (int col = 0; col < C; col++) {
            if constexpr (GRP) {
              x[col][0] = xst[(col * E + e) * S::kBW + k];
              x[col][1] = xst[(col * E + e + 1) * S::kBW + k];
            } else {
              x[col][0] = xst[(e * C + col) * S::kBW + k];
              x[col][1] = xst[((e + 1) * C + col) * S::kBW + k];
            }
          }
          const uint64_t ysa0 = shoup_factor8_np(ya0, p, np, delta), ysb0 = shoup_factor8_np(yb0, p, np, delta);
          const uint64_t ysa1 = shoup_factor8_np(ya1, p, np, delta), ysb1 = shoup_factor8_np(yb1, p, np, delta);
#pragma unroll
          for (int col = 0; col < C; col++) {
            const uint64_t x0 = x[col][0], x1 = x[col][1];
            st_v2(tb + (((0 * C + col) * (E / 2) + ep) * kW + k) * 2, shoup_lazy_np(x0, ya0, ysa0, np),
                  shoup_lazy_np(x1, ya1, ysa1, np));
            st_v2(tb + (((1 * C + col) * (E / 2) + ep) * kW + k) * 2, shoup_lazy_np(x0, yb0, ysb0, np),
                  shoup_lazy_np(x1, yb1, ysb1, np));
          }
        }
      } else {
#pragma unroll
        for (int it = 0; it < IPT; it++) {
          const int item = ct + it * kComputeThreads;
          const int k = item % kW, ep = item / kW, e = 2 * ep;
          const uint64_t ya0 = qst[(e * 2 + 0) * S::kBW + k], yb0 = qst[(e * 2 + 1) * S::kBW + k];
          const uint64_t ya1 = qst[(e * 2 + 2) * S::kBW + k], yb1 = qst[(e * 2 + 3) * S::kBW + k];
          const uint64_t ysa0 = shoup_factor8_np(ya0, p, np, delta), ysb0 = shoup_factor8_np(yb0, p, np, delta);
          const uint64_t ysa1 = shoup_factor8_np(ya1, p, np, delta), ysb1 = shoup_factor8_np(yb1, p, np, delta);
          const uint64_t x0 = xst[e * S::kBW + k], x1 = xst[(e + 1) * S::kBW + k];
          sts_v2(tb + (ep * kW + k) * 2, shoup_lazy_np(x0, ya0, ysa0, np), shoup_lazy_np(x1, ya1, ysa1, np));
          sts_v2(tb + (((E / 2) + ep) * kW + k) * 2, shoup_lazy_np(x0, yb0, ysb0, np), shoup_lazy_np(x1, yb1, ysb1, np));
        }
      }
      mbar_arrive(empty + s);
      mbar_arrive(tfull + b);
    }
  } else {
    // ---- chain warps: strictly in-order accumulation ---------------------------------
    const int u = threadIdx.x - 32 - kComputeThreads;  // (half, column, coefficient)
    if (u >= S::kChainThreads) return;
    const int h = u / (C * kW), col = (u / kW) % C, k = u % kW;
    uint64_t rop = 0;
    for (uint32_t t = 0; t < tiles; ++t) {
      const int b = (int)(t % TB);
      if (!mbar_wait(tfull + b, (t / TB) & 1, lim)) {
        ok = false;
        break;
      }
      const uint64_t *tb = terms + b * S::kT + ((h * C + col) * (E / 2) * kW + k) * 2;
      const uint64_t left = sh.n_i - (uint64_t)t * E;
      if (left >= (uint64_t)E) {
        // Terms come in batches of kB slot pairs; batch i+1 is requested before batch i
        // is accumulated, so only the 64-bit add/compare/subtract is on the serial path.
        constexpr int kB = 4;
        static_assert((E / 2) % kB == 0, "batches must divide the tile");
        uint64_t cur[2 * kB], nxt[2 * kB];
#pragma unroll
        for (int j = 0; j < kB; j++) lds_v2(tb + j * kW * 2, cur[2 * j], cur[2 * j + 1]);
#pragma unroll
        for (int e0 = 0; e0 < E / 2; e0 += kB) {
          if (e0 + kB < E / 2) {
#pragma unroll
            for (int j = 0; j < kB; j++) lds_v2(tb + (e0 + kB + j) * kW * 2, nxt[2 * j], nxt[2 * j + 1]);
          }
#pragma unroll
          for (int j = 0; j < 2 * kB; j++) {
            const uint64_t w = rop + cur[j];
            rop = w >= p ? w - p : w;
          }
#pragma unroll
          for (int j = 0; j < 2 * kB; j++) cur[j] = nxt[j];
        }
      } else {
        for (int e = 0; e < (int)left; e++) {
          const uint64_t w = rop + tb[((e / 2) * kW) * 2 + (e & 1)];
          rop = w >= p ? w - p : w;
        }
      }
      mbar_arrive(tempty + b);
    }
    const uint64_t mN = (uint64_t)sh.m * sh.N;
    if constexpr (GRP) {
      const uint64_t grp = g * C + col;  // one poly per element
      if (ok && grp < sh.groups && k0 + k < (int)sh.N) out[(grp * 2 + h) * mN + (uint64_t)c * sh.N + k0 + k] = rop;
    } else {
      const uint64_t cp = cp0 + col;
      if (ok && cp < sh.P && k0 + k < (int)sh.N) out[((g * sh.P + cp) * 2 + h) * mN + (uint64_t)c * sh.N + k0 + k] = rop;
    }
  }
  if (!ok) {
    *(volatile int *)status = kStatusWaitTimeout;
    __threadfence_system();
  }
}

// Two CTAs per SM for the narrow poly-column tiles (shared memory allows it), one for the
// wide ones; group-column tiles as many as their shared memory allows, up to three (the
// register budget then leaves them unspilled).
template <int W, int C, int E, int NS, int TB, int IPT, bool GRP>
constexpr int min_blocks() {
  using S = Cfg<W, C, E, NS, TB, IPT, GRP>;
  if constexpr (GRP) {
    constexpr size_t by_smem = (size_t)227 * 1024 / (S::kBytes + 1024);
    return by_smem >= 3 ? 3 : (by_smem == 2 ? 2 : 1);
  }
  return (C <= 2 && S::kThreads <= 640) ? 2 : 1;
}

// One query: tensor maps as grid constants.  Grid: x = group (GRP: block of C groups).
template <int W, int C, int E, int NS, int TB, int IPT, bool GRP>
__global__ void __launch_bounds__(Cfg<W, C, E, NS, TB, IPT, GRP>::kThreads, min_blocks<W, C, E, NS, TB, IPT, GRP>())
    reply_tma_kernel(const __grid_constant__ CUtensorMap tm_db, const __grid_constant__ CUtensorMap tm_q,
                     uint64_t *__restrict__ out, const LevelShape sh,
                     const DevModuli dm, int *status) {
  reply_tile<W, C, E, NS, TB, IPT, GRP>(&tm_db, &tm_q, out, blockIdx.x, sh, dm, status);
}

// Several tasks of one level shape (a batch of queries): each task's tensor maps and
// output come from a descriptor table in global memory.  Grid: x = group * tasks + task,
// so the CTAs of all queries that read the same DB tile run side by side and share it
// through L2.
template <int W, int C, int E, int NS, int TB, int IPT, bool GRP>
__global__ void __launch_bounds__(Cfg<W, C, E, NS, TB, IPT, GRP>::kThreads, min_blocks<W, C, E, NS, TB, IPT, GRP>())
    reply_tma_tasks_kernel(const ReplyTask *__restrict__ tasks, const uint32_t ntasks, const LevelShape sh,
                           const DevModuli dm, int *status) {
  const uint32_t t = blockIdx.x % ntasks;
  reply_tile<W, C, E, NS, TB, IPT, GRP>(&tasks[t].tm_db, &tasks[t].tm_q, tasks[t].out,
                                        blockIdx.x / ntasks, sh, dm, status);
}

// Tensor maps of one task for tile shape (W, C, E); GRP tiles load one poly column per
// group box.
template <int W, int C, int E, bool GRP>
bool encode_task(const uint64_t *db, const uint64_t *query, uint64_t n_real, uint64_t P, uint64_t n_i,
                 const ParamSet &ps, CUtensorMap *tm_db, CUtensorMap *tm_q) {
  const uint64_t N = ps.N, m = ps.m;
  const uint64_t db_dims[4] = {N, m, P, n_real};
  const uint64_t db_strides[3] = {N * 8, m * N * 8, P * m * N * 8};
  constexpr uint32_t kBW = (W % 4 == 0) ? W : W + 2;  // as Cfg::kBW
  const uint32_t db_box[4] = {kBW, 1, GRP ? 1u : (uint32_t)C, (uint32_t)E};
  const uint64_t q_dims[4] = {N, m, 2, n_i};
  const uint64_t q_strides[3] = {N * 8, m * N * 8, 2 * m * N * 8};
  const uint32_t q_box[4] = {kBW, 1, 2, (uint32_t)E};
  return encode_tensor_map_u64_4d(tm_db, db, db_dims, db_strides, db_box) &&
         encode_tensor_map_u64_4d(tm_q, query, q_dims, q_strides, q_box);
}

template <int W, int C, int E, int NS, int TB, int IPT, bool GRP>
cudaError_t launch_c(const ReplyLevelArgs &a, const ParamSet &ps, const DevModuli &dm, uint64_t groups,
                     cudaStream_t stream, int *status) {
  CUtensorMap tm_db, tm_q;
  if (!encode_task<W, C, E, GRP>(a.db, a.query, a.n_real, a.P, a.n_i, ps, &tm_db, &tm_q))
    return cudaErrorInvalidValue;
  using S = Cfg<W, C, E, NS, TB, IPT, GRP>;
  auto kern = reply_tma_kernel<W, C, E, NS, TB, IPT, GRP>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::kBytes);
  if (e != cudaSuccess) return e;
  if (GRP && (a.P != 1 || ((groups + C - 1) / C * C + 1) * a.n_i >= (1ull << 31))) return cudaErrorInvalidValue;
  const uint32_t col_blocks = GRP ? 1 : (uint32_t)((a.P + C - 1) / C);
  const uint64_t blocks = GRP ? (groups + C - 1) / C : groups;
  LevelShape sh{a.n_real, a.P, a.n_i, ps.N, ps.m, col_blocks, groups, a.wait_test};
  if (blocks > 0x7fffffffull || (uint64_t)ps.m * col_blocks > 65535) return cudaErrorInvalidValue;
  dim3 grid((unsigned)blocks, (ps.N + W - 1) / W, (unsigned)(ps.m * col_blocks));
  kern<<<grid, S::kThreads, S::kBytes, stream>>>(tm_db, tm_q, a.out, sh, dm, status);
  return cudaGetLastError();
}

template <int W, int C, int E, int NS, int TB, int IPT, bool GRP>
cudaError_t launch_tasks_c(const uint64_t *const *db, const uint64_t *const *query, uint64_t *const *out,
                           uint32_t ntasks, uint64_t n_real,
                           uint64_t P, uint64_t groups, uint64_t n_i, const ParamSet &ps, const DevModuli &dm,
                           ReplyTask *host_tasks, ReplyTask *dev_tasks, cudaStream_t stream, int *status) {
  for (uint32_t t = 0; t < ntasks; t++) {
    if (!encode_task<W, C, E, GRP>(db[t], query[t], n_real, P, n_i, ps, &host_tasks[t].tm_db, &host_tasks[t].tm_q)) {
      fprintf(stderr, "xpir_b200: tensor maps refused for task %u (database %p, query %p, %llu real, P %llu, n_i %llu)\n",
              t, (const void *)db[t], (const void *)query[t], (unsigned long long)n_real, (unsigned long long)P,
              (unsigned long long)n_i);
      return cudaErrorInvalidValue;
    }
    host_tasks[t].out = out[t];
  }
  cudaError_t e = cudaMemcpyAsync(dev_tasks, host_tasks, ntasks * sizeof(ReplyTask), cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return e;
  using S = Cfg<W, C, E, NS, TB, IPT, GRP>;
  auto kern = reply_tma_tasks_kernel<W, C, E, NS, TB, IPT, GRP>;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::kBytes);
  if (e != cudaSuccess) return e;
  if (GRP && (P != 1 || ((groups + C - 1) / C * C + 1) * n_i >= (1ull << 31))) return cudaErrorInvalidValue;
  const uint32_t col_blocks = GRP ? 1 : (uint32_t)((P + C - 1) / C);
  const uint64_t blocks = GRP ? (groups + C - 1) / C : groups;
  LevelShape sh{n_real, P, n_i, ps.N, ps.m, col_blocks, groups};
  if (blocks * ntasks > 0x7fffffffull || (uint64_t)ps.m * col_blocks > 65535) return cudaErrorInvalidValue;
  dim3 grid((unsigned)(blocks * ntasks), (ps.N + W - 1) / W, (unsigned)(ps.m * col_blocks));
  kern<<<grid, S::kThreads, S::kBytes, stream>>>(dev_tasks, ntasks, sh, dm, status);
  return cudaGetLastError();
}

typedef cudaError_t (*SingleFn)(const ReplyLevelArgs &, const ParamSet &, const DevModuli &, uint64_t, cudaStream_t,
                                int *);
typedef cudaError_t (*TasksFn)(const uint64_t *const *, const uint64_t *const *, uint64_t *const *, uint32_t, uint64_t, uint64_t, uint64_t, uint64_t, const ParamSet &,
                               const DevModuli &, ReplyTask *, ReplyTask *, cudaStream_t, int *);
struct TileEntry {
  TileShape shape;
  SingleFn single;
  TasksFn tasks;
  const void *single_kernel, *tasks_kernel;
};

#define XPIR_TILE_G(W, C, E, NS, TB, IPT, GRP)                                                              \
  {                                                                                                        \
    {W, C, E, NS, TB, IPT, GRP}, &launch_c<W, C, E, NS, TB, IPT, GRP>, &launch_tasks_c<W, C, E, NS, TB, IPT, GRP>, \
        (const void *)&reply_tma_kernel<W, C, E, NS, TB, IPT, GRP>,                                          \
        (const void *)&reply_tma_tasks_kernel<W, C, E, NS, TB, IPT, GRP>                                     \
  }
#define XPIR_TILE(W, C, E, NS, TB, IPT) XPIR_TILE_G(W, C, E, NS, TB, IPT, false)

// Every compiled tile shape.  Entries 0..2 are the one-column shapes for grids of at
// most two CTAs per SM, picked by slice width (two slot pairs per compute thread);
// entry 3 is the one-column shape for larger grids (one slot pair per thread: more
// warps per SM); entries 4..5 are further one-column shapes for the autotuner; then one
// entry per column count 2..8 with 16-coefficient slices, and the same with 8 (twice
// the CTAs, for levels whose grid would not fill the GPU).  E, NS, TB come from timing
// sweeps on B200 over E in {16..128}, NS in {2..8}, TB in {2, 4, 8}.  The last entries
// but one take C groups as columns, for one-poly levels with several groups (the
// recursion's first level): each query tile and Shoup factor then serves C groups, which
// cuts the L2-to-SM query traffic and the factor work by C and puts 2*C*W chains in each
// CTA.  The last is a seven-column narrow shape with 64-slot tiles for grids of at most
// one CTA per SM.
const TileEntry kTiles[] = {
    XPIR_TILE(14, 1, 64, 3, 2, 2),
    XPIR_TILE(16, 1, 64, 3, 2, 2),
    XPIR_TILE(8, 1, 128, 3, 2, 2),
    XPIR_TILE(16, 1, 64, 3, 2, 1),
    XPIR_TILE(16, 1, 32, 4, 4, 1),
    XPIR_TILE(32, 1, 32, 3, 4, 1),
    XPIR_TILE(16, 2, 32, 3, 2, 1),
    XPIR_TILE(16, 3, 16, 4, 2, 1),
    XPIR_TILE(16, 4, 16, 3, 2, 1),
    XPIR_TILE(16, 5, 16, 3, 2, 1),
    XPIR_TILE(16, 6, 16, 3, 2, 1),
    XPIR_TILE(16, 7, 16, 3, 2, 1),
    XPIR_TILE(16, 8, 16, 3, 2, 1),
    XPIR_TILE(8, 2, 32, 3, 2, 1),
    XPIR_TILE(8, 3, 32, 3, 2, 1),
    XPIR_TILE(8, 4, 32, 3, 2, 1),
    XPIR_TILE(8, 5, 32, 3, 2, 1),
    XPIR_TILE(8, 6, 32, 3, 2, 1),
    XPIR_TILE(8, 7, 32, 3, 2, 1),
    XPIR_TILE(8, 8, 32, 3, 2, 1),
    XPIR_TILE_G(16, 2, 32, 3, 2, 1, true),
    XPIR_TILE_G(16, 4, 16, 3, 2, 1, true),
    XPIR_TILE_G(16, 8, 16, 3, 2, 1, true),
    XPIR_TILE_G(8, 4, 32, 3, 2, 1, true),
    XPIR_TILE_G(8, 8, 32, 3, 2, 1, true),
    XPIR_TILE(8, 7, 64, 3, 2, 1),
};
constexpr int kTileCount = sizeof(kTiles) / sizeof(kTiles[0]);
constexpr int kFirstColumnTile = 6;        // entry of C = 2, W = 16
constexpr int kFirstNarrowColumnTile = 13;  // entry of C = 2, W = 8
constexpr int kFirstGroupTile = 20;        // group columns (one-poly levels)
constexpr int kGroupTile = 21;             // default for one-poly levels with >= 4 groups: C = 4, W = 16
constexpr int kManyCtaTile = 3;      // one column, grids beyond two CTAs per SM
constexpr int kDeepNarrow7Tile = 25;  // C = 7, W = 8 with 64-slot tiles: twice the compute warps

// Streaming multiprocessors of the current device (cached per device).
int sm_count() {
  static int cache[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cache[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cache[dev] = n;
  }
  return cache[dev];
}

}  // namespace

bool reply_level_supported(const ParamSet &ps, uint64_t n_real, uint64_t n_i, uint64_t groups) {
  for (uint32_t c = 0; c < ps.m; c++)
    if (!shoup_factor8_ok(ps.mod[c].p)) return false;
  // TMA coordinates are 32-bit signed.
  return ps.N % 16 == 0 && n_real < (1ull << 31) && groups * n_i + 256 < (1ull << 31);
}

// One-poly levels with at least four groups (per task) take group columns.  Otherwise
// one column per CTA: every CTA of a level does the same work (its slice width W times
// the level's slots), and an SM's CTAs share its issue slots, so a grid of at most two
// CTAs per SM takes about ceil(CTAs / SMs) * W.  The default takes the slice width that
// minimises this (the widest on ties: longer TMA rows), e.g. W=14 for N=2048 and two
// moduli (294 CTAs on 148 SMs against 256 for W=16, which leaves 40 SMs with half the
// work of the others).
int default_tile(uint64_t P, uint32_t N, uint32_t m, uint64_t groups, uint64_t ntasks) {
  const uint64_t sms = (uint64_t)sm_count();
  const uint64_t ctas_per_slice = groups * ntasks;
  if (P == 1 && groups >= (uint64_t)kTiles[kGroupTile].shape.C) return kGroupTile;
  if (P > 1) {
    // C columns per CTA; 16- or 8-coefficient slices by the same cost (the 1,000 x 12 KB
    // level at N=1024: 64 CTAs of W=16 against 128 of W=8, which run 1.7x faster).
    const int C = (int)(P >= 8 ? 8 : P);
    const int wide = kFirstColumnTile + C - 2, narrow = kFirstNarrowColumnTile + C - 2;
    if (N == 0) return wide;
    const uint64_t col_blocks = (P + C - 1) / C;
    const uint64_t ctas16 = ctas_per_slice * m * ((N + 15) / 16) * col_blocks;
    const uint64_t ctas8 = ctas_per_slice * m * ((N + 7) / 8) * col_blocks;
    const uint64_t cost16 = (ctas16 + sms - 1) / sms * 16, cost8 = (ctas8 + sms - 1) / sms * 8;
    if (cost8 >= cost16) return wide;
    // A narrow seven-column grid with at most one CTA per SM: the 64-slot tile's eight
    // compute warps (220 KB of shared memory, one CTA per SM) beat two 32-slot tiles' four
    // (the 1,000 x 12 KB level at N=1024: 47 against 54 us).
    return (C == 7 && ctas8 <= sms) ? kDeepNarrow7Tile : narrow;
  }
  int best = 1;
  uint64_t best_cost = ~0ull, best_ctas = 0;
  for (int t : {1, 0, 2}) {
    const uint64_t W = (uint64_t)kTiles[t].shape.W;
    const uint64_t ctas = ctas_per_slice * m * ((N + W - 1) / W);
    const uint64_t cost = (ctas + sms - 1) / sms * W;
    if (cost < best_cost) {
      best = t;
      best_cost = cost;
      best_ctas = ctas;
    }
  }
  // Several waves of CTAs: the SMs stay evenly loaded anyway, and more warps per CTA
  // hide more latency (measured on the recursive and batched workloads).
  return best_ctas > 2 * sms ? kManyCtaTile : best;
}

std::vector<int> tile_candidates(uint64_t P) {
  if (P <= 1) {
    std::vector<int> c = {0, 1, 2, 3, 4, 5};
    for (int t = kFirstGroupTile; t < kTileCount; t++)
      if (kTiles[t].shape.grp) c.push_back(t);
    return c;
  }
  // several columns per CTA (query tiles shared), 16- or 8-coefficient slices, or
  // one column per CTA
  const int C = (int)(P >= 8 ? 8 : P);
  if (C == 7) return {kFirstColumnTile + C - 2, kFirstNarrowColumnTile + C - 2, kDeepNarrow7Tile, kManyCtaTile};
  return {kFirstColumnTile + C - 2, kFirstNarrowColumnTile + C - 2, kManyCtaTile};
}

TileShape tile_shape(int tile) { return kTiles[tile].shape; }

// Whether a tile can run a level with P polys per element: poly columns no wider than P
// (at most 8), group columns only for one-poly levels.
bool tile_fits(int tile, uint64_t P) {
  if (tile < 0 || tile >= kTileCount) return false;
  if (kTiles[tile].shape.grp) return P == 1;
  return kTiles[tile].shape.C <= (int)(P > 8 ? 8 : P);
}
int tile_count() { return kTileCount; }

cudaError_t launch_reply_tasks(const uint64_t *const *db, const uint64_t *const *query, uint64_t *const *out,
                               uint32_t ntasks, uint64_t n_real,
                               uint64_t P, uint64_t n_groups, uint64_t n_i, const ParamSet &ps, const DevModuli &dm,
                               ReplyTask *host_tasks, ReplyTask *dev_tasks, cudaStream_t stream, uint32_t *launches,
                               int *status, int tile, bool write_idle) {
  if (ntasks == 0) return cudaSuccess;
  const uint64_t ct_words = 2ull * ps.m * ps.N;
  const uint64_t active = active_groups(n_real, n_i, n_groups);
  if (active < n_groups && write_idle) {
    for (uint32_t t = 0; t < ntasks; t++) {
      cudaError_t e = cudaMemsetAsync(out[t] + active * P * ct_words, 0,
                                      (n_groups - active) * P * ct_words * sizeof(uint64_t), stream);
      if (e != cudaSuccess) return e;
    }
  }
  if (active == 0) return cudaSuccess;
  if (!reply_level_supported(ps, n_real, n_i, active * ntasks)) return cudaErrorNotSupported;
  if (!tile_fits(tile, P)) tile = default_tile(P, ps.N, ps.m, active, ntasks);
  if (launches) (*launches)++;
  return kTiles[tile].tasks(db, query, out, ntasks, n_real, P, active, n_i, ps, dm, host_tasks, dev_tasks,
                            stream, status);
}

cudaError_t launch_reply_level(const ReplyLevelArgs &a, const ParamSet &ps, const DevModuli &dm,
                               cudaStream_t stream, uint32_t *launches, int *status, int tile) {
  const uint64_t ct_words = 2ull * ps.m * ps.N;
  // Groups whose every slot is past the real elements accumulate only zero terms from
  // a zero start: their replies are exactly zero.  Only groups with data are launched.
  const uint64_t active = active_groups(a.n_real, a.n_i, a.n_groups);
  if (active < a.n_groups && a.write_idle) {
    cudaError_t e = cudaMemsetAsync(a.out + active * a.P * ct_words, 0,
                                    (a.n_groups - active) * a.P * ct_words * sizeof(uint64_t), stream);
    if (e != cudaSuccess) return e;
  }
  if (active == 0) return cudaSuccess;
  if (!reply_level_supported(ps, a.n_real, a.n_i, active)) return cudaErrorNotSupported;
  if (launches) (*launches)++;
  if (!tile_fits(tile, a.P)) tile = default_tile(a.P, ps.N, ps.m, active, 1);
  return kTiles[tile].single(a, ps, dm, active, stream, status);
}

// Loads every compiled reply kernel on the current device (lazy module loading would
// otherwise do it, and reserve their device memory, at each one's first launch).
cudaError_t preload_reply_kernels() {
  cudaFuncAttributes fa;
  for (const TileEntry &t : kTiles) {
    cudaError_t e = cudaFuncGetAttributes(&fa, t.single_kernel);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, t.tasks_kernel);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace xpir
