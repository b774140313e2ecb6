// C ABI of the B200 reply engine (include/xpir_b200.h).
//
// Host orchestration only: parameter set and tables (params.cpp), then the kernels of
// import.cu and reply.cu ordered on the context's stream.  No CPU compute path exists:
// every call either runs on the GPU or returns an error status.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <mutex>
#include <set>
#include <vector>

#include "xpir_b200.h"
#include "handles.h"
#include "kernels.h"
#include "params.h"

using namespace xpir;

namespace {

thread_local cudaError_t g_last_cuda = cudaSuccess;

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return XPIR_B200_OK;
  g_last_cuda = e;
  (void)cudaGetLastError();  // clear the sticky-free error state where possible
  if (e == cudaErrorMemoryAllocation) return XPIR_B200_ERR_NOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice || e == cudaErrorInsufficientDriver)
    return XPIR_B200_ERR_NODEV;
  return XPIR_B200_ERR_CUDA;
}

#define XPIR_TRY(expr)                         \
  do {                                         \
    const cudaError_t e_ = (expr);             \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

int grow(void **buf, size_t *have, size_t need) {
  if (need <= *have) return XPIR_B200_OK;
  if (*buf) {
    XPIR_TRY(cudaFree(*buf));
    *buf = nullptr;
    *have = 0;
  }
  XPIR_TRY(cudaMalloc(buf, need));
  *have = need;
  return XPIR_B200_OK;
}

bool mul_ok(uint64_t a, uint64_t b, uint64_t *out) {
  if (a != 0 && b > UINT64_MAX / a) return false;
  *out = a * b;
  return true;
}

ParamSet with_bits(const ParamSet &base, uint32_t b) {
  ParamSet ps = base;
  ps.b = b;
  return ps;
}

}  // namespace

void xpir::note_cuda_error(cudaError_t e) {
  if (e != cudaSuccess) g_last_cuda = e;
}

extern "C" {

const char *xpir_b200_version(void) { return "xpir_b200 0.1 (sm_100a)"; }

const char *xpir_b200_strerror(int status) {
  switch (status) {
    case XPIR_B200_OK: return "ok";
    case XPIR_B200_ERR_ARG: return "invalid argument or unsupported shape";
    case XPIR_B200_ERR_NOMEM: return "out of device or pinned host memory";
    case XPIR_B200_ERR_CUDA: return "CUDA runtime error";
    case XPIR_B200_ERR_NODEV: return "no usable CUDA device";
    case XPIR_B200_ERR_STATE: return "call out of order";
    case XPIR_B200_ERR_TIMEOUT: return "a device-side bounded wait expired";
    default: return "unknown status";
  }
}

const char *xpir_b200_last_cuda_error(void) { return cudaGetErrorName(g_last_cuda); }

int xpir_b200_device_count(int *count) {
  if (!count) return XPIR_B200_ERR_ARG;
  *count = 0;
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) {
    *count = 0;
    return cuda_status(e);
  }
  return XPIR_B200_OK;
}

int32_t xpir_b200_bits_per_coeff(uint32_t N, uint32_t m, uint32_t k, uint64_t n0) {
  if (!valid_shape(N, m) || n0 == 0) return 0;
  return bits_per_coeff(N, m, k, n0);
}

uint64_t xpir_b200_polys_per_element(uint64_t element_bytes, uint32_t alpha, uint32_t b, uint32_t N) {
  return polys_for_bits(8ull * alpha * element_bytes, b, N);
}

uint64_t xpir_b200_reply_count(uint64_t element_bytes, uint32_t alpha, uint32_t d, uint32_t b, uint32_t N,
                               uint32_t m) {
  return reply_count(element_bytes, alpha, d, b, N, m);
}

uint64_t xpir_b200_ciphertext_bytes(uint32_t N, uint32_t m) { return ciphertext_bytes(N, m); }

uint64_t xpir_b200_modulus(uint32_t i) { return i < kMaxModuli ? kModuli[i] : 0; }

int xpir_b200_ctx_create(xpir_b200_ctx **out, int device, uint32_t N, uint32_t m) {
  if (!out) return XPIR_B200_ERR_ARG;
  *out = nullptr;
  if (!valid_shape(N, m)) return XPIR_B200_ERR_ARG;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    (void)cudaGetLastError();
    return XPIR_B200_ERR_NODEV;
  }
  if (device < 0 || device >= count) return XPIR_B200_ERR_NODEV;
  auto *ctx = new (std::nothrow) xpir_b200_ctx();
  if (!ctx) return XPIR_B200_ERR_NOMEM;
  ctx->device = device;
  std::vector<uint64_t> tables;
  if (!build_params(N, m, 1, &ctx->ps, &tables)) {
    delete ctx;
    return XPIR_B200_ERR_ARG;
  }
  int rc = cuda_status(cudaSetDevice(device));
  // Load every engine kernel and place the no-allocation scratch on this device now, so
  // that no later call loads a module (module loading reserves device memory).
  if (rc == XPIR_B200_OK) rc = cuda_status(preload_import_kernels());
  if (rc == XPIR_B200_OK) rc = cuda_status(preload_reply_kernels());
  if (rc == XPIR_B200_OK) rc = cuda_status(prepare_noalloc_scratch(device));
  if (rc == XPIR_B200_OK) rc = cuda_status(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  if (rc == XPIR_B200_OK) rc = cuda_status(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  if (rc == XPIR_B200_OK) rc = cuda_status(cudaEventCreateWithFlags(&ctx->query_copied, cudaEventDisableTiming));
  if (rc == XPIR_B200_OK) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    rc = cuda_status(cudaMemPoolCreate(&ctx->pool, &props));
  }
  if (rc == XPIR_B200_OK) {
    uint64_t keep = UINT64_MAX;
    rc = cuda_status(cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  if (rc == XPIR_B200_OK) rc = cuda_status(cudaMalloc(&ctx->d_tables, tables.size() * sizeof(uint64_t)));
  if (rc == XPIR_B200_OK)
    rc = cuda_status(cudaMemcpy(ctx->d_tables, tables.data(), tables.size() * sizeof(uint64_t),
                                cudaMemcpyHostToDevice));
  if (rc == XPIR_B200_OK) rc = cuda_status(cudaHostAlloc(&ctx->status_host, sizeof(int), cudaHostAllocMapped));
  if (rc == XPIR_B200_OK) {
    *ctx->status_host = 0;
    rc = cuda_status(cudaHostGetDevicePointer((void **)&ctx->status_dev, ctx->status_host, 0));
  }
  if (rc != XPIR_B200_OK) {
    xpir_b200_ctx_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return XPIR_B200_OK;
}

int xpir_b200_ctx_destroy(xpir_b200_ctx *ctx) {
  if (!ctx) return XPIR_B200_ERR_ARG;
  if (ctx->servers.load() > 0) return XPIR_B200_ERR_STATE;  // a server's lane still runs on it
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (xpir_b200_db *db : ctx->dbs) {
    cudaFree(db->d_polys);
    delete db;
  }
  ctx->dbs.clear();
  cudaFree(ctx->d_tables);
  cudaFree(ctx->ws_query);
  cudaFree(ctx->ws_a);
  cudaFree(ctx->ws_b);
  cudaFree(ctx->tasks_dev);
  if (ctx->tasks_host) cudaFreeHost(ctx->tasks_host);
  ctx->plans.clear();
  if (ctx->status_host) cudaFreeHost(ctx->status_host);
  for (auto &pair : ctx->timing_ev)
    for (cudaEvent_t ev : pair)
      if (ev) cudaEventDestroy(ev);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  if (ctx->query_copied) cudaEventDestroy(ctx->query_copied);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
  delete ctx;
  return XPIR_B200_OK;
}

int xpir_b200_ctx_stream(xpir_b200_ctx *ctx, void **stream) {
  if (!ctx || !stream) return XPIR_B200_ERR_ARG;
  *stream = (void *)ctx->stream;
  return XPIR_B200_OK;
}

int xpir_b200_ctx_synchronize(xpir_b200_ctx *ctx) {
  if (!ctx) return XPIR_B200_ERR_ARG;
  XPIR_TRY(cudaSetDevice(ctx->device));
  XPIR_TRY(cudaStreamSynchronize(ctx->stream));
  return XPIR_B200_OK;
}

int xpir_b200_ctx_set_wait_test(xpir_b200_ctx *ctx, uint32_t spin_limit, int32_t withhold_tile) {
  if (!ctx || withhold_tile < -1) return XPIR_B200_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->wait_test.spin_limit = spin_limit;
  ctx->wait_test.withhold_tile = withhold_tile;
  return XPIR_B200_OK;
}

int xpir_b200_ctx_set_kernel_timing(xpir_b200_ctx *ctx, int on) {
  if (!ctx) return XPIR_B200_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  if (on) {
    XPIR_TRY(cudaSetDevice(ctx->device));
    for (auto &pair : ctx->timing_ev)
      for (cudaEvent_t &ev : pair)
        if (!ev) XPIR_TRY(cudaEventCreate(&ev));
    for (uint32_t l = 0; l < XPIR_B200_MAX_LEVELS; l++) {
      ctx->reply_ms[l] = 0;
      ctx->reply_timed[l] = 0;
    }
    ctx->import_ms = 0;
    ctx->import_timed = 0;
  }
  ctx->timing = on != 0;
  return XPIR_B200_OK;
}

int xpir_b200_ctx_kernel_time(xpir_b200_ctx *ctx, double *reply_ms, uint64_t *reply_launches, double *import_ms,
                              uint64_t *import_launches) {
  if (!ctx) return XPIR_B200_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  for (uint32_t l = 0; l < XPIR_B200_MAX_LEVELS; l++) {
    if (reply_ms) reply_ms[l] = ctx->reply_ms[l];
    if (reply_launches) reply_launches[l] = ctx->reply_timed[l];
  }
  if (import_ms) *import_ms = ctx->import_ms;
  if (import_launches) *import_launches = ctx->import_timed;
  return XPIR_B200_OK;
}

int xpir_b200_ctx_launch_count(xpir_b200_ctx *ctx, uint64_t *count) {
  if (!ctx || !count) return XPIR_B200_ERR_ARG;
  *count = ctx->launches;
  return XPIR_B200_OK;
}

int xpir_b200_db_import(xpir_b200_ctx *ctx, const void *elements, uint64_t nb_elements, uint64_t element_bytes,
                        uint64_t element_stride, uint32_t alpha, uint32_t b, int src_on_device,
                        xpir_b200_db **out) {
  if (!ctx || !out || !elements || nb_elements == 0 || element_bytes == 0 || alpha == 0) return XPIR_B200_ERR_ARG;
  if (element_stride < element_bytes || b == 0 || b > 4 * 56) return XPIR_B200_ERR_ARG;
  *out = nullptr;
  std::lock_guard<std::mutex> lock(ctx->mu);
  XPIR_TRY(cudaSetDevice(ctx->device));
  const ParamSet ps = with_bits(ctx->ps, b);
  const uint64_t groups = (nb_elements + alpha - 1) / alpha;
  uint64_t agg_bits;
  if (!mul_ok(8ull * alpha, element_bytes, &agg_bits)) return XPIR_B200_ERR_ARG;
  const uint64_t P = polys_for_bits(agg_bits, b, ps.N);
  uint64_t words, tmp;
  if (!mul_ok(groups, P, &tmp) || !mul_ok(tmp, (uint64_t)ps.m * ps.N, &words)) return XPIR_B200_ERR_ARG;
  const uint64_t src_bytes = (nb_elements - 1) * element_stride + element_bytes;

  auto *db = new (std::nothrow) xpir_b200_db();
  if (!db) return XPIR_B200_ERR_NOMEM;
  db->ctx = ctx;
  db->id = next_db_id();
  db->n_agg = groups;
  db->P = P;
  db->b = b;
  db->alpha = alpha;
  db->element_bytes = element_bytes;
  cudaError_t e = cudaMalloc(&db->d_polys, words * sizeof(uint64_t));
  if (e != cudaSuccess) {
    delete db;
    return cuda_status(e);
  }
  const uint8_t *src = (const uint8_t *)elements;
  void *staging = nullptr;
  if (!src_on_device) {
    e = cudaMalloc(&staging, src_bytes);
    if (e == cudaSuccess) e = cudaMemcpyAsync(staging, elements, src_bytes, cudaMemcpyHostToDevice, ctx->stream);
    src = (const uint8_t *)staging;
  }
  if (e == cudaSuccess) {
    const AggSource as{src, nb_elements, element_bytes, element_stride, alpha};
    e = launch_import(as, groups, P, ps, make_dev_moduli(ps), ctx->d_tables, db->d_polys, ctx->stream);
    ctx->launches++;
  }
  if (staging) {
    cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = e2;
    cudaFree(staging);
  }
  if (e != cudaSuccess) {
    cudaFree(db->d_polys);
    delete db;
    return cuda_status(e);
  }
  ctx->dbs.insert(db);
  *out = db;
  return XPIR_B200_OK;
}

int xpir_b200_db_free(xpir_b200_db *db) {
  if (!db) return XPIR_B200_ERR_ARG;
  xpir_b200_ctx *ctx = db->ctx;
  std::lock_guard<std::mutex> lock(ctx->mu);
  if (!ctx->dbs.erase(db)) return XPIR_B200_ERR_ARG;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  drop_plans_of(ctx, db->id);
  cudaFree(db->d_polys);
  delete db;
  return XPIR_B200_OK;
}

int xpir_b200_db_info(const xpir_b200_db *db, uint64_t *nb_aggregated, uint64_t *polys_per_element,
                      uint32_t *bits_per_coeff, uint64_t *device_bytes) {
  if (!db) return XPIR_B200_ERR_ARG;
  if (nb_aggregated) *nb_aggregated = db->n_agg;
  if (polys_per_element) *polys_per_element = db->P;
  if (bits_per_coeff) *bits_per_coeff = db->b;
  if (device_bytes) *device_bytes = db->n_agg * db->P * db->ctx->ps.m * db->ctx->ps.N * sizeof(uint64_t);
  return XPIR_B200_OK;
}

int xpir_b200_db_export(const xpir_b200_db *db, uint64_t *host_out, uint64_t capacity_words) {
  if (!db || !host_out) return XPIR_B200_ERR_ARG;
  const uint64_t words = db->n_agg * db->P * db->ctx->ps.m * db->ctx->ps.N;
  if (capacity_words < words) return XPIR_B200_ERR_ARG;
  std::lock_guard<std::mutex> lock(db->ctx->mu);
  XPIR_TRY(cudaSetDevice(db->ctx->device));
  XPIR_TRY(cudaMemcpyAsync(host_out, db->d_polys, words * 8, cudaMemcpyDeviceToHost, db->ctx->stream));
  XPIR_TRY(cudaStreamSynchronize(db->ctx->stream));
  return XPIR_B200_OK;
}

int xpir_b200_reply(xpir_b200_ctx *ctx, const xpir_b200_db *db, uint32_t d, const uint32_t *n, const void *query,
                    int query_on_device, void *replies, uint64_t capacity_bytes, int out_on_device,
                    uint64_t *nb_replies) {
  if (!ctx || !db || !n || !query || !replies || d == 0 || d > XPIR_B200_MAX_LEVELS) return XPIR_B200_ERR_ARG;
  if (db->ctx != ctx) return XPIR_B200_ERR_ARG;
  uint64_t slots = 1, total_ct = 0;
  for (uint32_t i = 0; i < d; i++) {
    if (n[i] == 0 || !mul_ok(slots, n[i], &slots)) return XPIR_B200_ERR_ARG;
    total_ct += n[i];
  }
  // The reference sizes its grid as prod(n) and writes one entry per aggregated element.
  if (slots < db->n_agg) return XPIR_B200_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  XPIR_TRY(cudaSetDevice(ctx->device));
  const ParamSet ps = with_bits(ctx->ps, db->b);
  const DevModuli dm = make_dev_moduli(ps);
  const uint64_t mN = (uint64_t)ps.m * ps.N, ct_words = 2 * mN, ct_bytes = ct_words * 8;

  // Work out every level's shape first so that the workspaces grow at most once.
  uint64_t Ps[XPIR_B200_MAX_LEVELS], groups[XPIR_B200_MAX_LEVELS];
  size_t need_a = 0, need_b = 0;
  Ps[0] = db->P;
  for (uint32_t lvl = 0; lvl < d; lvl++) {
    groups[lvl] = 1;
    for (uint32_t j = lvl + 1; j < d; j++) groups[lvl] *= n[j];
    uint64_t rep_bytes;
    if (!mul_ok(groups[lvl] * Ps[lvl], ct_bytes, &rep_bytes)) return XPIR_B200_ERR_ARG;
    if (lvl + 1 < d) {
      need_a = rep_bytes > need_a ? rep_bytes : need_a;
      Ps[lvl + 1] = polys_for_bits(Ps[lvl] * ct_bytes * 8, ps.b, ps.N);
      const uint64_t next_bytes = groups[lvl] * Ps[lvl + 1] * mN * 8;
      need_b = next_bytes > need_b ? next_bytes : need_b;
    }
  }
  const uint64_t final_count = Ps[d - 1];
  const uint64_t final_bytes = final_count * ct_bytes;
  if (capacity_bytes < final_bytes) return XPIR_B200_ERR_ARG;
  if (!out_on_device) need_a = final_bytes > need_a ? final_bytes : need_a;
  int rc;
  if ((rc = grow(&ctx->ws_a, &ctx->ws_a_bytes, need_a)) != XPIR_B200_OK) return rc;
  if ((rc = grow(&ctx->ws_b, &ctx->ws_b_bytes, need_b)) != XPIR_B200_OK) return rc;

  const uint64_t *dq = (const uint64_t *)query;
  const bool split_copy = !query_on_device && d > 1;
  // Every return waits for the copy stream, so that no copy from the caller's query is
  // left in flight (on success it has long finished: level 2 waited for it).
  struct CopyGuard {
    cudaStream_t s;
    bool on;
    ~CopyGuard() {
      if (on) cudaStreamSynchronize(s);
    }
  } copy_guard{ctx->copy_stream, split_copy};
  if (!query_on_device) {
    if ((rc = grow(&ctx->ws_query, &ctx->ws_query_bytes, total_ct * ct_bytes)) != XPIR_B200_OK) return rc;
    // The first level's ciphertexts on the context's stream; the other levels' on the copy
    // stream, so that the first level's reply runs while they cross PCIe (the level loop
    // waits for them before level 2).
    const uint64_t first = (uint64_t)n[0] * ct_bytes;
    XPIR_TRY(cudaMemcpyAsync(ctx->ws_query, query, first, cudaMemcpyHostToDevice, ctx->stream));
    if (split_copy) {
      XPIR_TRY(cudaMemcpyAsync((char *)ctx->ws_query + first, (const char *)query + first,
                               (total_ct - n[0]) * ct_bytes, cudaMemcpyHostToDevice, ctx->copy_stream));
      XPIR_TRY(cudaEventRecord(ctx->query_copied, ctx->copy_stream));
    }
    dq = (const uint64_t *)ctx->ws_query;
  }

  const uint64_t *in = db->d_polys;
  uint64_t in_real = db->n_agg;
  *ctx->status_host = 0;
  // Event pairs of this call (kernel timing): [2*lvl] the level's reply, [2*lvl+1] the
  // re-import after it; a pair is read only when its launch was recorded.
  bool timed[2 * XPIR_B200_MAX_LEVELS] = {};
  auto time_begin = [&](uint32_t k) -> cudaError_t {
    return ctx->timing ? cudaEventRecord(ctx->timing_ev[k][0], ctx->stream) : cudaSuccess;
  };
  auto time_end = [&](uint32_t k, uint32_t launched) -> cudaError_t {
    if (!ctx->timing || launched == 0) return cudaSuccess;
    timed[k] = true;
    return cudaEventRecord(ctx->timing_ev[k][1], ctx->stream);
  };
  for (uint32_t lvl = 0; lvl < d; lvl++) {
    const bool last = lvl + 1 == d;
    uint64_t *rep = (last && out_on_device) ? (uint64_t *)replies : (uint64_t *)ctx->ws_a;
    uint32_t launched = 0;
    if (lvl == 1 && split_copy) XPIR_TRY(cudaStreamWaitEvent(ctx->stream, ctx->query_copied, 0));
    ReplyLevelArgs a{in, in_real, Ps[lvl], groups[lvl], n[lvl], dq, rep};
    a.write_idle = last;
    a.wait_test = ctx->wait_test;
    const uint64_t active = active_groups(in_real, n[lvl], groups[lvl]);
    XPIR_TRY(time_begin(2 * lvl));
    const cudaError_t le = launch_reply_level(a, ps, dm, ctx->stream, &launched, ctx->status_dev,
                                              tuned_tile(ctx, Ps[lvl], n[lvl], groups[lvl]));
    if (le == cudaErrorNotSupported) return XPIR_B200_ERR_ARG;
    XPIR_TRY(le);
    XPIR_TRY(time_end(2 * lvl, launched));
    ctx->launches += launched;
    dq += (uint64_t)n[lvl] * ct_words;
    if (last) break;
    // Level replies -> next level's database: element e's Ps[lvl] ciphertexts are one
    // contiguous bit stream (no inverse NTT, as the reference).
    // Groups past `active` replied exactly zero (and were not written out).
    const AggSource as{(const uint8_t *)rep, groups[lvl], Ps[lvl] * ct_bytes, Ps[lvl] * ct_bytes, 1};
    const ImportRows rows{1, groups[lvl], active};
    launched = 0;
    XPIR_TRY(time_begin(2 * lvl + 1));
    XPIR_TRY(launch_import(as, groups[lvl], Ps[lvl + 1], ps, dm, ctx->d_tables, (uint64_t *)ctx->ws_b,
                           ctx->stream, &rows, &launched));
    XPIR_TRY(time_end(2 * lvl + 1, launched));
    ctx->launches += launched;
    in = (const uint64_t *)ctx->ws_b;
    in_real = groups[lvl];
  }
  if (!out_on_device)
    XPIR_TRY(cudaMemcpyAsync(replies, ctx->ws_a, final_bytes, cudaMemcpyDeviceToHost, ctx->stream));
  XPIR_TRY(cudaStreamSynchronize(ctx->stream));
  for (uint32_t k = 0; k < 2 * d; k++) {
    if (!timed[k]) continue;
    float ms = 0;
    XPIR_TRY(cudaEventElapsedTime(&ms, ctx->timing_ev[k][0], ctx->timing_ev[k][1]));
    if (k % 2 == 0) {
      ctx->reply_ms[k / 2] += ms;
      ctx->reply_timed[k / 2]++;
    } else {
      ctx->import_ms += ms;
      ctx->import_timed++;
    }
  }
  if (*(volatile int *)ctx->status_host != 0) return XPIR_B200_ERR_TIMEOUT;
  if (nb_replies) *nb_replies = final_count;
  return XPIR_B200_OK;
}

}  // extern "C"
