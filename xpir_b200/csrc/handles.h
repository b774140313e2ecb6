// Definitions of the opaque C-ABI handles (internal to the engine library).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <set>

#include "params.h"

struct xpir_b200_db;

struct xpir_b200_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  xpir::ParamSet ps;           // b is set per database
  uint64_t *d_tables = nullptr;
  std::mutex mu;
  uint64_t launches = 0;
  // grow-only workspaces (device)
  void *ws_query = nullptr;
  size_t ws_query_bytes = 0;
  void *ws_a = nullptr;  // level replies
  size_t ws_a_bytes = 0;
  void *ws_b = nullptr;  // re-imported level databases
  size_t ws_b_bytes = 0;
  int *status_host = nullptr;  // kernel status word (mapped pinned memory)
  int *status_dev = nullptr;
  std::set<xpir_b200_db *> dbs;  // databases imported through this context
};

struct xpir_b200_db {
  xpir_b200_ctx *ctx = nullptr;
  uint64_t *d_polys = nullptr;
  uint64_t n_agg = 0;
  uint64_t P = 0;
  uint32_t b = 0;
  uint32_t alpha = 1;
  uint64_t element_bytes = 0;
};

