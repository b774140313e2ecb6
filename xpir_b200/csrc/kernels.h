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
//
// With `rows`, the groups elements form rows->rows rows of rows->per_row, and in each row
// only the first rows->active elements carry data: the rest are known all-zero bit
// streams (level replies of groups that had no real slot, which are exactly zero).  All
// their polys import to one constant poly per modulus -- not zero: the lazy butterflies
// turn zeros into multiples of p -- which a fill kernel computes once per CTA and
// broadcasts instead of running the import on each.  *launches (if given) is increased
// by the kernels launched.
struct ImportRows {
  uint64_t rows, per_row, active;
};

// The secret key's Shoup factors (sks = floor(sk * 2^64 / p), sk words below p) for
// query generation and extraction, computed on the device on `stream`.
cudaError_t launch_key_shoup(const uint64_t *sk, uint64_t *sks, uint32_t N, uint32_t m, const DevModuli &dm,
                             cudaStream_t stream);

// Lets `kernel` take up to the current device's opt-in maximum of dynamic shared memory.
// For a kernel whose shared memory depends on the parameter set (import, extraction,
// query generation), every caller sets this same value: contexts of different parameter
// sets launch it from several threads, and a per-launch size set by one thread between
// another thread's setting and launch made that launch fail (cudaErrorInvalidValue).
cudaError_t allow_max_dynamic_smem(const void *kernel);

cudaError_t launch_import(const AggSource &src, uint64_t groups, uint64_t P, const ParamSet &ps,
                          const DevModuli &dm, const uint64_t *tables, uint64_t *out, cudaStream_t stream,
                          const ImportRows *rows = nullptr, uint32_t *launches = nullptr);

// Test support for the reply kernel's bounded waits (xpir_b200_ctx_set_wait_test): a
// shorter limit for the waits of the consumer warps and of the copy producer's ring, and
// a tile whose copies the producer never issues (-1: none), so that the waits for that
// tile run out, the kernel records kStatusWaitTimeout and returns.  The producer's final
// wait for its own copies in flight keeps the full limit.
struct WaitTest {
  uint32_t spin_limit = 0;  // 0: the default limit (sm100.cuh kSpinLimit)
  int32_t withhold_tile = -1;
};

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
  // Whether the replies of groups without a real slot (exactly zero) are written out.
  // A level whose replies only feed the next level's import (which knows they are zero,
  // see ImportRows) skips it.
  bool write_idle = true;
  WaitTest wait_test;
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
  uint64_t *out;
};

// A compiled tile shape of the reply kernel: W coefficients per slice, C columns per
// CTA, E slots per tile, NS pipeline stages, TB term buffers, IPT slot pairs per
// compute thread; the columns are polys of one element, or with grp groups of a
// one-poly level.
struct TileShape {
  int W, C, E, NS, TB, IPT;
  bool grp;
};
// Index of the default shape for a level with P polys per element, degree N, m moduli,
// `groups` active groups per task and `ntasks` tasks in the launch.
int default_tile(uint64_t P, uint32_t N, uint32_t m, uint64_t groups, uint64_t ntasks);
// Shapes the autotuner may try for a level with P polys per element.
std::vector<int> tile_candidates(uint64_t P);
TileShape tile_shape(int tile);
int tile_count();
// Whether a tile can run a level with P polys per element.
bool tile_fits(int tile, uint64_t P);

// `ntasks` reply levels of the same shape (n_real, P, n_groups, n_i), one per query,
// in one launch.  `host_tasks` (pinned, ntasks entries) is filled here and copied to
// `dev_tasks` on `stream` before the launch.  tile < 0 picks the default shape.
cudaError_t launch_reply_tasks(const uint64_t *const *db, const uint64_t *const *query, uint64_t *const *out,
                               uint32_t ntasks, uint64_t n_real,
                               uint64_t P, uint64_t n_groups, uint64_t n_i, const ParamSet &ps, const DevModuli &dm,
                               ReplyTask *host_tasks, ReplyTask *dev_tasks, cudaStream_t stream, uint32_t *launches,
                               int *status, int tile, bool write_idle = true);

// Groups of a level that hold at least one real element (the others reply exactly zero).
inline uint64_t active_groups(uint64_t n_real, uint64_t n_i, uint64_t n_groups) {
  const uint64_t a = n_i == 0 ? 0 : (n_real + n_i - 1) / n_i;
  return a < n_groups ? a : n_groups;
}

// Whether the reply kernel supports this level shape (moduli with the fast Shoup-factor
// path, degree a multiple of 16, 32-bit TMA coordinates).
bool reply_level_supported(const ParamSet &ps, uint64_t n_real, uint64_t n_i, uint64_t groups);

// Load the import and reply kernels on the current device, so that no later launch
// loads a module (which reserves device memory).
cudaError_t preload_import_kernels();
cudaError_t preload_reply_kernels();
// Places the scratch array of xpir_b200_reply_noalloc on the current device (loading
// the module that holds it) and caches its device address (noalloc.cu).
cudaError_t prepare_noalloc_scratch(int device);

}  // namespace xpir
