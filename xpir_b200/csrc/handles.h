// Definitions of the opaque C-ABI handles (internal to the engine library).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <tuple>
#include <vector>

#include "kernels.h"
#include "params.h"
#include "xpir_b200.h"

struct xpir_b200_db;
struct BatchPlan;  // batch.cu

// Tile-shape choices made by xpir_b200_autotune, keyed by level shape (P, n_i, groups).
typedef std::map<std::tuple<uint64_t, uint64_t, uint64_t>, int> TuneTable;

struct xpir_b200_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  // Host queries of recursive replies: the later levels' ciphertexts are copied on this
  // stream while the first level replies; the event marks the end of that copy.
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t query_copied = nullptr;
  xpir::ParamSet ps;           // b is set per database
  uint64_t *d_tables = nullptr;
  std::mutex mu;
  std::atomic<uint64_t> launches{0};  // engine kernels launched (also counted off the lock)
  std::atomic<int> servers{0};         // servers with a lane on this context
  cudaError_t last_error = cudaSuccess;  // the last CUDA error of a batch on this context
  // grow-only workspaces (device)
  void *ws_query = nullptr;
  size_t ws_query_bytes = 0;
  void *ws_a = nullptr;  // level replies
  size_t ws_a_bytes = 0;
  void *ws_b = nullptr;  // re-imported level databases
  size_t ws_b_bytes = 0;
  void *tasks_dev = nullptr;   // task table of uncaptured batches (device copy)
  void *tasks_host = nullptr;  // and its pinned staging copy
  size_t tasks_cap = 0;        // entries of both
  // Stream-ordered pool of the client-side entry points' per-call buffers (query
  // generation, extraction): it keeps freed memory for the next call (release threshold
  // UINT64_MAX), so that a call after the first maps no new device memory.
  cudaMemPool_t pool = nullptr;
  int *status_host = nullptr;  // kernel status word (mapped pinned memory)
  int *status_dev = nullptr;
  std::set<xpir_b200_db *> dbs;  // databases imported through this context
  TuneTable tuned;
  uint64_t tune_epoch = 0;  // bumped by every autotune (invalidates captured batches)
  xpir::WaitTest wait_test;  // test support of the bounded waits (xpir_b200_ctx_set_wait_test)
  // Kernel timing (xpir_b200_ctx_set_kernel_timing): an event pair around each level's
  // reply launch and each re-import of xpir_b200_reply, summed after the call's sync.
  bool timing = false;
  cudaEvent_t timing_ev[2 * XPIR_B200_MAX_LEVELS][2] = {};
  double reply_ms[XPIR_B200_MAX_LEVELS] = {}, import_ms = 0;
  uint64_t reply_timed[XPIR_B200_MAX_LEVELS] = {}, import_timed = 0;
  std::vector<std::shared_ptr<BatchPlan>> plans;  // captured batches (batch.cu)
};

// Tile shape for a level shape: the autotuned one if any, else -1 (default).
inline int tuned_tile(const xpir_b200_ctx *ctx, uint64_t P, uint64_t n_i, uint64_t groups) {
  auto it = ctx->tuned.find(std::make_tuple(P, n_i, groups));
  return it == ctx->tuned.end() ? -1 : it->second;
}

struct xpir_b200_db {
  xpir_b200_ctx *ctx = nullptr;
  uint64_t id = 0;  // unique per import in this process (never reused, unlike the address)
  uint64_t *d_polys = nullptr;
  uint64_t n_agg = 0;
  uint64_t P = 0;
  uint32_t b = 0;
  uint32_t alpha = 1;
  uint64_t element_bytes = 0;
};

struct xpir_b200_request;

namespace xpir {
// Records a CUDA error as the calling thread's xpir_b200_last_cuda_error().
void note_cuda_error(cudaError_t e);
}  // namespace xpir

namespace xpir {

// A fresh database id (1, 2, ...): captured batches are keyed by it, so a database
// imported at the address of a freed one never replays the freed one's graph.
inline uint64_t next_db_id() {
  static std::atomic<uint64_t> counter{0};
  return ++counter;
}

// Drops the captured batches that read database `db_id` (batch.cu).  The caller holds
// ctx->mu and has synchronised the context's stream.
void drop_plans_of(xpir_b200_ctx *ctx, uint64_t db_id);

// Supplies the workspace of an uncaptured batch: device buffers of at least `a` bytes
// (level replies) and `b` bytes (re-imported level databases), valid in stream order on
// the context's stream until the batch call returns.
typedef std::function<cudaError_t(size_t a, size_t b, void **pa, void **pb)> WorkspaceFn;

// xpir_b200_reply_batch with an optional workspace supplier (null: the context's own
// cached workspaces).  Used by the serving loop to draw workspaces from its budgeted pool.
int reply_batch_impl(xpir_b200_ctx *ctx, xpir_b200_request *reqs, uint32_t count, int use_graph,
                     const WorkspaceFn *workspace);

}  // namespace xpir
