// Kernel launchers of the B200 reply engine (device code in import.cu / reply.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "params.h"

namespace xpir {

// A database viewed the way the reference reads it for import: nb_elements elements of
// element_bytes bytes (element i at base + i*element_stride), grouped alpha at a time
// into aggregated elements of alpha*element_bytes bytes.  The last group, when short,
// follows DBHandler::readAggregatedStream's reused-buffer behaviour
// (pir/dbhandlers/DBHandler.cpp:3-26).
struct AggSource {
  const uint8_t *base;
  uint64_t nb_elements;
  uint64_t element_bytes;
  uint64_t element_stride;
  uint32_t alpha;
};

// Per-modulus constants the device needs, by value.
struct DevModuli {
  uint64_t p[kMaxModuli];
  uint64_t shoup_k[kMaxModuli];
  uint64_t shoup_delta[kMaxModuli];
  uint64_t crt[kMaxModuli][4];
  uint64_t crt_shoup[kMaxModuli][4];
};

DevModuli make_dev_moduli(const ParamSet &ps);

// Import: for every aggregated element s < groups and poly j < P, bit-split + CRT +
// phi-twist + forward NTT into out[(s*P + j)][m][N].  groups = ceil(nb/alpha),
// P = polys_for_bits(8*alpha*element_bytes, b, N).  `tables` is the device copy of the
// ParamSet tables.  Returns a CUDA error code.
cudaError_t launch_import(const AggSource &src, uint64_t groups, uint64_t P, const ParamSet &ps,
                          const DevModuli &dm, const uint64_t *tables, uint64_t *out, cudaStream_t stream);

// One recursion level of the reply (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:511-595):
// for group g < n_groups and poly cp < P, the in-order lazy Shoup accumulation over the
// n_i slots of the group; slot q reads DB element g*n_i + q, an all-zero element when
// that index is >= n_real.  out: [n_groups][P][2][m][N].
struct ReplyLevelArgs {
  const uint64_t *db;     // [n_real][P][m][N]
  uint64_t n_real;
  uint64_t P;
  uint64_t n_groups;
  uint64_t n_i;
  const uint64_t *query;  // [n_i][2][m][N]
  uint64_t *out;
  // The query's Shoup factors (same layout), from launch_query_factors, or null to derive
  // them in the kernel.  Used by one-poly levels (P = 1).
  const uint64_t *query_factors = nullptr;
};
// `status` is a device-visible int that a kernel sets to a nonzero KernelStatus when one
// of its bounded waits gives up (sm100.cuh); the caller clears and reads it.
cudaError_t launch_reply_level(const ReplyLevelArgs &a, const ParamSet &ps, const DevModuli &dm,
                               cudaStream_t stream, uint32_t *launches, int *status, int tile = -1);

// One task of a multi-task reply-level launch: the DB level of the task viewed as
// [element][poly][modulus][coefficient], its query level as [slot][half][modulus][coefficient],
// and its output [group][poly][half][modulus][coefficient].  Built on the host, copied
// to device memory, read by the kernel (TMA takes the tensor maps' global addresses).
struct alignas(128) ReplyTask {
  CUtensorMap tm_db;
  CUtensorMap tm_q;
  CUtensorMap tm_qf;  // query factors (tiles that read them)
  uint64_t *out;
};

// A compiled tile shape of the reply kernel: W coefficients per slice, C poly columns
// per CTA, E slots per tile, NS pipeline stages, TB term buffers, IPT slot pairs per
// compute thread, pre: reads precomputed query factors.
struct TileShape {
  int W, C, E, NS, TB, IPT;
  bool pre;
};
// Index of the default shape for a level with P polys per element, degree N, m moduli
// and `ctas_per_slice` CTAs per (coefficient slice, modulus) (active groups x tasks).
int default_tile(uint64_t P, uint32_t N, uint32_t m, uint64_t ctas_per_slice);
// Shapes the autotuner may try for a level with P polys per element.
std::vector<int> tile_candidates(uint64_t P);
TileShape tile_shape(int tile);
int tile_count();

// `ntasks` reply levels of the same shape (n_real, P, n_groups, n_i), one per query,
// in one launch.  `host_tasks` (pinned, ntasks entries) is filled here and copied to
// `dev_tasks` on `stream` before the launch.  tile < 0 picks the default shape.
cudaError_t launch_reply_tasks(const uint64_t *const *db, const uint64_t *const *query,
                               const uint64_t *const *factors, uint64_t *const *out, uint32_t ntasks, uint64_t n_real,
                               uint64_t P, uint64_t n_groups, uint64_t n_i, const ParamSet &ps, const DevModuli &dm,
                               ReplyTask *host_tasks, ReplyTask *dev_tasks, cudaStream_t stream, uint32_t *launches,
                               int *status, int tile);

// Groups of a level that hold at least one real element (the others reply exactly zero).
inline uint64_t active_groups(uint64_t n_real, uint64_t n_i, uint64_t n_groups) {
  const uint64_t a = n_i == 0 ? 0 : (n_real + n_i - 1) / n_i;
  return a < n_groups ? a : n_groups;
}

// Whether a level should read precomputed query factors: one poly per element and at
// least four groups sharing each query slot, so that deriving every factor once (one
// memory-bound pass) replaces deriving it once per group inside the reply kernel.
inline bool level_uses_factors(uint64_t P, uint64_t active) { return P == 1 && active >= 4; }

// The Shoup factors of n_ct query ciphertexts into `factors` (same layout and size).
cudaError_t launch_query_factors(const uint64_t *query, uint64_t *factors, uint64_t n_ct, const ParamSet &ps,
                                 const DevModuli &dm, cudaStream_t stream, uint32_t *launches);

// Whether the reply kernel supports this level shape (moduli with the fast Shoup-factor
// path, degree a multiple of 16, 32-bit TMA coordinates).
bool reply_level_supported(const ParamSet &ps, uint64_t n_real, uint64_t n_i, uint64_t groups);

}  // namespace xpir
