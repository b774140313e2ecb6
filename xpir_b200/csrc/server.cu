// Serving loop: continuous batching of queries over resident databases, admission by a
// device-memory budget, one lane per context (an uploading thread with its copy stream
// and a computing thread with the context's stream), so that batches of different
// parameter sets overlap on the GPU and, within a lane, one batch's copies overlap the
// previous batch's replies.  See admission.h for the
// queueing rules; this file runs a batch on the engine.
//
// No counterpart in the reference, whose server answers one query per session and
// streams replies as they appear (apps/server/PIRSession.cpp:467-565).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <mutex>
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
  // set by the upload stage, used by the compute stage
  void *dq = nullptr, *dr = nullptr;
  cudaEvent_t uploaded = nullptr;  // on the batch's first query only
  int upload_status = 0;
  cudaError_t cuda_error = cudaSuccess;  // the CUDA error behind an XPIR_B200_ERR_CUDA status
};

}  // namespace

struct xpir_b200_server {
  std::vector<xpir_b200_ctx *> ctxs;
  std::vector<cudaMemPool_t> pools;         // one stream-ordered pool per lane, on its device
  std::vector<cudaStream_t> copy_streams;   // host-to-device copies and pulls, beside the context's stream
  std::unique_ptr<xpir::Admission> adm;
};

namespace {

// A CUDA error of a served batch, on stderr (the query's status carries it too).
void report(const char *where, uint32_t lane, cudaError_t e) {
  fprintf(stderr, "xpir_b200 server: %s failed on lane %u: %s\n", where, lane, cudaGetErrorName(e));
}

int status_of_error(cudaError_t e) {
  return e == cudaErrorMemoryAllocation ? XPIR_B200_ERR_NOMEM : XPIR_B200_ERR_CUDA;
}

// A lane is a two-stage pipeline (admission.h).  Every device buffer of a batch
// (queries, replies, recursion workspace) comes from the lane's stream-ordered pool and
// goes back to it in stream order, so no stage synchronises the device or holds memory
// beyond the footprints admission reserved; other lanes keep running meanwhile.
//
// The host-to-device copies of all streams complete in the order they were issued on the
// copy engine, so one multi-GB query copied by it holds every other lane's copies (and
// through them their replies) until it has crossed PCIe: 235 ms for a 12.9 GB query.
// Queries of kPullBytes or more whose host buffer is mapped pinned memory are therefore
// pulled over PCIe by a small kernel instead (about 50 GB/s with 8,192 threads against the
// copy engine's 55), which leaves the copy engine to the other lanes' queries.
constexpr uint64_t kPullBytes = 256ull << 20;
constexpr int kPullBlocks = 32, kPullThreads = 256;

__global__ void __launch_bounds__(kPullThreads) pull_host_kernel(const uint4 *__restrict__ src,
                                                                 uint4 *__restrict__ dst, uint64_t n16) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // Four 16-byte loads in flight per thread: PCIe round trips are microseconds long.
  for (; i + 3 * stride < n16; i += 4 * stride) {
    const uint4 a = src[i], b = src[i + stride], c = src[i + 2 * stride], d = src[i + 3 * stride];
    dst[i] = a;
    dst[i + stride] = b;
    dst[i + 2 * stride] = c;
    dst[i + 3 * stride] = d;
  }
  for (; i < n16; i += stride) dst[i] = src[i];
}

// The address, on `device`, of a host buffer that is pinned memory mapped for that
// device, or null (pageable memory, or pinned on behalf of another device).
const void *mapped_device_address(const void *host, int device) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, host) != cudaSuccess) {
    (void)cudaGetLastError();
    return nullptr;
  }
  return at.type == cudaMemoryTypeHost && at.device == device ? at.devicePointer : nullptr;
}

// Stage 1, on the admitting thread: the batch's query and reply buffers and the queries'
// host-to-device copies, on the lane's copy stream; an event marks their completion.
void upload_batch(xpir_b200_server *srv, uint32_t lane, std::vector<xpir::Job *> &batch) {
  xpir_b200_ctx *ctx = srv->ctxs[lane];
  cudaStream_t cs = srv->copy_streams[lane];
  cudaError_t e = cudaSetDevice(ctx->device);
  for (size_t i = 0; i < batch.size(); i++) {
    auto *q = (ServedQuery *)batch[i]->payload.get();
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&q->dq, q->query_bytes ? q->query_bytes : 256, srv->pools[lane], cs);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&q->dr, q->reply_bytes ? q->reply_bytes : 256, srv->pools[lane], cs);
    if (e != cudaSuccess) continue;
    const void *mapped = q->query_bytes >= kPullBytes ? mapped_device_address(q->host_query, ctx->device) : nullptr;
    if (mapped && (((uintptr_t)mapped | (uintptr_t)q->dq | q->query_bytes) & 15) == 0) {
      pull_host_kernel<<<kPullBlocks, kPullThreads, 0, cs>>>((const uint4 *)mapped, (uint4 *)q->dq,
                                                            q->query_bytes / 16);
      e = cudaGetLastError();
      ctx->launches++;
    } else {
      e = cudaMemcpyAsync(q->dq, q->host_query, q->query_bytes, cudaMemcpyHostToDevice, cs);
    }
  }
  auto *q0 = (ServedQuery *)batch[0]->payload.get();
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&q0->uploaded, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(q0->uploaded, cs);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    report("upload", lane, e);
    for (auto *j : batch) {
      auto *q = (ServedQuery *)j->payload.get();
      q->upload_status = status_of_error(e);
      q->cuda_error = e;
    }
  }
}

// Stage 2, on the lane's second thread: once the copies are done, one batched reply on
// the context's stream (workspace from the pool), the replies copied back, buffers freed.
void compute_batch(xpir_b200_server *srv, uint32_t lane, std::vector<xpir::Job *> &batch) {
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
  auto *q0 = (ServedQuery *)batch[0]->payload.get();
  cudaError_t e = cudaSetDevice(ctx->device);
  const int upload = q0->upload_status;
  if (e == cudaSuccess && upload == XPIR_B200_OK) e = cudaStreamWaitEvent(st, q0->uploaded, 0);
  std::vector<xpir_b200_request> reqs(batch.size());
  for (size_t i = 0; i < batch.size(); i++) {
    auto *q = (ServedQuery *)batch[i]->payload.get();
    xpir_b200_request &r = reqs[i];
    memset(&r, 0, sizeof(r));
    r.db = q->db;
    r.d = q->d;
    memcpy(r.n, q->n, sizeof(r.n));
    r.query = q->dq;
    r.replies = q->dr;
    r.capacity_bytes = q->reply_bytes;
  }
  const xpir::WorkspaceFn ws = [&](size_t a, size_t b, void **pa, void **pb) -> cudaError_t {
    const cudaError_t r = alloc(a, pa);
    return r == cudaSuccess ? alloc(b, pb) : r;
  };
  const bool run = e == cudaSuccess && upload == XPIR_B200_OK;
  if (run) xpir::reply_batch_impl(ctx, reqs.data(), (uint32_t)reqs.size(), 0, &ws);
  for (size_t i = 0; i < batch.size(); i++) {
    auto *q = (ServedQuery *)batch[i]->payload.get();
    int s = run ? reqs[i].status : (upload != XPIR_B200_OK ? upload : status_of_error(e));
    if (!run && upload == XPIR_B200_OK) q->cuda_error = e;
    if (run && s == XPIR_B200_ERR_CUDA) q->cuda_error = ctx->last_error;
    if (i == 0 && !run && upload == XPIR_B200_OK) report("wait for the upload", lane, e);
    if (i == 0 && run && s == XPIR_B200_ERR_CUDA) report("batched reply", lane, ctx->last_error);
    if (s == XPIR_B200_OK) {
      q->nb_replies = reqs[i].nb_replies;
      const cudaError_t ce = cudaMemcpyAsync(q->host_replies, q->dr, q->reply_bytes, cudaMemcpyDeviceToHost, st);
      if (ce != cudaSuccess) {
        s = XPIR_B200_ERR_CUDA;
        q->cuda_error = ce;
        report("reply copy to the host", lane, ce);
      }
    }
    batch[i]->status = s;
  }
  for (size_t i = 0; i < batch.size(); i++) {
    auto *q = (ServedQuery *)batch[i]->payload.get();
    if (q->dq) cudaFreeAsync(q->dq, st);
    if (q->dr) cudaFreeAsync(q->dr, st);
    q->dq = q->dr = nullptr;
  }
  for (void *p : held) cudaFreeAsync(p, st);
  const cudaError_t se = cudaStreamSynchronize(st);
  if (se != cudaSuccess) report("batch synchronisation", lane, se);
  if (se != cudaSuccess)
    for (auto *j : batch) {
      j->status = XPIR_B200_ERR_CUDA;
      ((ServedQuery *)j->payload.get())->cuda_error = se;
    }
  if (q0->uploaded) cudaEventDestroy(q0->uploaded);
  q0->uploaded = nullptr;
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
  for (uint32_t lvl = 0; lvl + 1 < d; lvl++) {
    uint64_t groups = 1;
    for (uint32_t j = lvl + 1; j < d; j++) groups *= n[j];
    const uint64_t P2 = xpir::polys_for_bits(P * ct_bytes * 8, db->b, ctx->ps.N);
    ws = std::max(ws, groups * P * ct_bytes + groups * P2 * mN * 8);
    P = P2;
  }
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
  for (uint32_t i = 0; i < nctx; i++) {
    cudaStream_t cs = nullptr;
    cudaError_t e = cudaSetDevice(ctxs[i]->device);
    // The highest priority: a pull kernel's few CTAs are placed ahead of the replies'
    // waiting CTAs (stream priority orders CTA scheduling, not copy-engine work).
    int least = 0, greatest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&cs, cudaStreamNonBlocking, greatest);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      for (cudaStream_t s2 : srv->copy_streams) cudaStreamDestroy(s2);
      for (cudaMemPool_t p : srv->pools) cudaMemPoolDestroy(p);
      delete srv;
      return XPIR_B200_ERR_CUDA;
    }
    srv->copy_streams.push_back(cs);
  }
  // Two batches in flight per lane: one uploading while the previous one computes.
  srv->adm.reset(new xpir::Admission(
      nctx, device_budget_bytes, max_batch,
      [srv](uint32_t lane, std::vector<xpir::Job *> &b) { upload_batch(srv, lane, b); },
      [srv](uint32_t lane, std::vector<xpir::Job *> &b) { compute_batch(srv, lane, b); }, 2));
  for (xpir_b200_ctx *c : srv->ctxs) c->servers++;
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
  if (status == XPIR_B200_ERR_CUDA) xpir::note_cuda_error(((ServedQuery *)j->payload.get())->cuda_error);
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
  srv->adm->stop(XPIR_B200_ERR_STATE);
  for (xpir_b200_ctx *c : srv->ctxs) c->servers--;
  for (cudaStream_t cs : srv->copy_streams) cudaStreamDestroy(cs);
  for (cudaMemPool_t p : srv->pools) cudaMemPoolDestroy(p);
  delete srv;
  return XPIR_B200_OK;
}

}  // extern "C"
