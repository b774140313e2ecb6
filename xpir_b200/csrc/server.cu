// Serving loop: continuous batching of queries over resident databases, admission by a
// device-memory budget, one lane (worker thread + the context's stream) per context, so
// that batches of different parameter sets overlap on the GPU.  See admission.h for the
// queueing rules; this file runs a batch on the engine.
//
// No counterpart in the reference, whose server answers one query per session and
// streams replies as they appear (apps/server/PIRSession.cpp:467-565).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "admission.h"
#include "handles.h"
#include "kernels.h"
#include "params.h"
#include "xpir_b200.h"

namespace {

struct ServedQuery {
  const xpir_b200_db *db = nullptr;
  uint32_t d = 0;
  uint32_t n[XPIR_B200_MAX_LEVELS] = {};
  const void *host_query = nullptr;  // caller's buffer, valid until the wait returns
  void *host_replies = nullptr;
  uint64_t query_bytes = 0, reply_bytes = 0, capacity = 0, nb_replies = 0;
};

}  // namespace

struct xpir_b200_server {
  std::vector<xpir_b200_ctx *> ctxs;
  std::vector<cudaMemPool_t> pools;  // one stream-ordered pool per lane, on its device
  std::unique_ptr<xpir::Admission> adm;
};

namespace {

// Runs one admitted batch of one lane.  Every device buffer of the batch (queries,
// replies, recursion workspace) comes from the lane's stream-ordered pool and goes back
// to it in stream order, so the batch neither synchronises the device nor holds memory
// beyond the footprints admission reserved for it; other lanes keep running meanwhile.
void run_batch(xpir_b200_server *srv, uint32_t lane, std::vector<xpir::Job *> &batch) {
  xpir_b200_ctx *ctx = srv->ctxs[lane];
  cudaStream_t st = ctx->stream;
  cudaMemPool_t pool = srv->pools[lane];
  std::vector<void *> held;
  auto alloc = [&](size_t bytes, void **p) -> cudaError_t {
    *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes ? bytes : 256, pool, st);
    if (e == cudaSuccess) held.push_back(*p);
    return e;
  };
  cudaError_t e = cudaSetDevice(ctx->device);
  std::vector<xpir_b200_request> reqs(batch.size());
  std::vector<void *> dr(batch.size(), nullptr);
  for (size_t i = 0; i < batch.size() && e == cudaSuccess; i++) {
    auto *q = (ServedQuery *)batch[i]->payload.get();
    void *dq = nullptr;
    e = alloc(q->query_bytes, &dq);
    if (e == cudaSuccess) e = alloc(q->reply_bytes, &dr[i]);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dq, q->host_query, q->query_bytes, cudaMemcpyHostToDevice, st);
    xpir_b200_request &r = reqs[i];
    memset(&r, 0, sizeof(r));
    r.db = q->db;
    r.d = q->d;
    memcpy(r.n, q->n, sizeof(r.n));
    r.query = dq;
    r.replies = dr[i];
    r.capacity_bytes = q->reply_bytes;
  }
  const xpir::WorkspaceFn ws = [&](size_t a, size_t b, size_t f, void **pa, void **pb, void **pf) -> cudaError_t {
    cudaError_t r = alloc(a, pa);
    if (r == cudaSuccess) r = alloc(b, pb);
    return r == cudaSuccess ? alloc(f, pf) : r;
  };
  if (e == cudaSuccess) xpir::reply_batch_impl(ctx, reqs.data(), (uint32_t)reqs.size(), 0, &ws);
  for (size_t i = 0; i < batch.size(); i++) {
    auto *q = (ServedQuery *)batch[i]->payload.get();
    int s = e == cudaSuccess ? reqs[i].status : (e == cudaErrorMemoryAllocation ? XPIR_B200_ERR_NOMEM : XPIR_B200_ERR_CUDA);
    if (s == XPIR_B200_OK) {
      q->nb_replies = reqs[i].nb_replies;
      if (cudaMemcpyAsync(q->host_replies, dr[i], q->reply_bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        s = XPIR_B200_ERR_CUDA;
    }
    batch[i]->status = s;
  }
  for (void *p : held) cudaFreeAsync(p, st);
  if (cudaStreamSynchronize(st) != cudaSuccess)
    for (auto *j : batch) j->status = XPIR_B200_ERR_CUDA;
}

// Device bytes a query holds while admitted: its query and reply buffers and its share
// of the batch's recursion workspace (level replies and re-imported level databases).
bool footprint_of(const xpir_b200_db *db, uint32_t d, const uint32_t *n, uint64_t *query_bytes,
                  uint64_t *reply_bytes, uint64_t *footprint) {
  const xpir_b200_ctx *ctx = db->ctx;
  const uint64_t mN = (uint64_t)ctx->ps.m * ctx->ps.N, ct_bytes = 2 * mN * 8;
  uint64_t slots = 1, nq = 0, P = db->P, ws = 0;
  for (uint32_t i = 0; i < d; i++) {
    if (n[i] == 0 || slots > UINT64_MAX / n[i]) return false;
    slots *= n[i];
    nq += n[i];
  }
  if (slots < db->n_agg) return false;
  uint64_t fws = 0, real = db->n_agg;
  for (uint32_t lvl = 0; lvl < d; lvl++) {
    uint64_t groups = 1;
    for (uint32_t j = lvl + 1; j < d; j++) groups *= n[j];
    if (xpir::level_uses_factors(P, xpir::active_groups(real, n[lvl], groups))) fws = std::max(fws, n[lvl] * ct_bytes);
    if (lvl + 1 == d) break;
    const uint64_t P2 = xpir::polys_for_bits(P * ct_bytes * 8, db->b, ctx->ps.N);
    ws = std::max(ws, groups * P * ct_bytes + groups * P2 * mN * 8);
    P = P2;
    real = groups;
  }
  ws += fws;
  *query_bytes = nq * ct_bytes;
  *reply_bytes = P * ct_bytes;
  *footprint = *query_bytes + *reply_bytes + ws;
  return true;
}

}  // namespace

extern "C" {

int xpir_b200_server_create(xpir_b200_server **out, xpir_b200_ctx *const *ctxs, uint32_t nctx,
                            uint64_t device_budget_bytes, uint32_t max_batch) {
  if (!out || !ctxs || nctx == 0 || device_budget_bytes == 0) return XPIR_B200_ERR_ARG;
  for (uint32_t i = 0; i < nctx; i++)
    if (!ctxs[i]) return XPIR_B200_ERR_ARG;
  auto *srv = new (std::nothrow) xpir_b200_server();
  if (!srv) return XPIR_B200_ERR_NOMEM;
  srv->ctxs.assign(ctxs, ctxs + nctx);
  // A private pool per lane that keeps freed memory for reuse (release threshold at
  // its maximum), so steady-state batches map no new memory.
  for (uint32_t i = 0; i < nctx; i++) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = ctxs[i]->device;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    uint64_t keep = UINT64_MAX;
    if (e == cudaSuccess) e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      if (pool) cudaMemPoolDestroy(pool);
      for (cudaMemPool_t p : srv->pools) cudaMemPoolDestroy(p);
      delete srv;
      return e == cudaErrorNoDevice || e == cudaErrorInvalidDevice ? XPIR_B200_ERR_NODEV : XPIR_B200_ERR_CUDA;
    }
    srv->pools.push_back(pool);
  }
  srv->adm.reset(new xpir::Admission(nctx, device_budget_bytes, max_batch,
                                     [srv](uint32_t lane, std::vector<xpir::Job *> &b) { run_batch(srv, lane, b); }));
  *out = srv;
  return XPIR_B200_OK;
}

int xpir_b200_server_submit(xpir_b200_server *srv, const xpir_b200_db *db, uint32_t d, const uint32_t *n,
                            const void *query, void *replies, uint64_t capacity_bytes, uint64_t *ticket) {
  if (!srv || !db || !n || !query || !replies || !ticket || d == 0 || d > XPIR_B200_MAX_LEVELS)
    return XPIR_B200_ERR_ARG;
  *ticket = 0;
  uint32_t lane = 0;
  while (lane < srv->ctxs.size() && srv->ctxs[lane] != db->ctx) lane++;
  if (lane == srv->ctxs.size()) return XPIR_B200_ERR_ARG;
  auto q = std::make_shared<ServedQuery>();
  if (!footprint_of(db, d, n, &q->query_bytes, &q->reply_bytes, &q->capacity)) return XPIR_B200_ERR_ARG;
  const uint64_t footprint = q->capacity;
  if (capacity_bytes < q->reply_bytes) return XPIR_B200_ERR_ARG;
  q->capacity = capacity_bytes;
  q->db = db;
  q->d = d;
  memcpy(q->n, n, d * sizeof(uint32_t));
  q->host_query = query;
  q->host_replies = replies;
  const uint64_t t = srv->adm->submit(lane, footprint, q);
  if (t == 0) return XPIR_B200_ERR_NOMEM;  // larger than the whole device budget
  *ticket = t;
  return XPIR_B200_OK;
}

int xpir_b200_server_wait(xpir_b200_server *srv, uint64_t ticket, int timeout_ms, uint64_t *nb_replies,
                          double *latency_s, double *queued_s) {
  if (!srv) return XPIR_B200_ERR_ARG;
  xpir::Job *j = srv->adm->wait(ticket, timeout_ms);
  if (!j) return XPIR_B200_ERR_STATE;  // unknown ticket or not done within the timeout
  const int status = j->status;
  if (nb_replies) *nb_replies = ((ServedQuery *)j->payload.get())->nb_replies;
  if (latency_s) *latency_s = j->t_done - j->t_submit;
  if (queued_s) *queued_s = j->t_admit - j->t_submit;
  srv->adm->release(ticket);
  return status;
}

int xpir_b200_server_footprint(const xpir_b200_db *db, uint32_t d, const uint32_t *n, uint64_t *bytes) {
  if (!db || !n || !bytes || d == 0 || d > XPIR_B200_MAX_LEVELS) return XPIR_B200_ERR_ARG;
  uint64_t qb, rb;
  return footprint_of(db, d, n, &qb, &rb, bytes) ? XPIR_B200_OK : XPIR_B200_ERR_ARG;
}

int xpir_b200_server_stats(xpir_b200_server *srv, uint64_t *completed, uint64_t *batches, uint64_t *max_batch,
                           uint64_t *peak_device_bytes) {
  if (!srv) return XPIR_B200_ERR_ARG;
  const xpir::AdmissionStats s = srv->adm->stats();
  if (completed) *completed = s.completed;
  if (batches) *batches = s.batches;
  if (max_batch) *max_batch = s.max_batch_seen;
  if (peak_device_bytes) *peak_device_bytes = s.peak_in_use;
  return XPIR_B200_OK;
}

int xpir_b200_server_destroy(xpir_b200_server *srv) {
  if (!srv) return XPIR_B200_ERR_ARG;
  srv->adm->stop();
  for (cudaMemPool_t p : srv->pools) cudaMemPoolDestroy(p);
  delete srv;
  return XPIR_B200_OK;
}

}  // extern "C"
