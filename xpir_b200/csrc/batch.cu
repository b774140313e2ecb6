// Batches of queries (xpir_b200_reply_batch), captured CUDA graphs of repeated batches,
// and the tile-shape autotuner (xpir_b200_autotune).
//
// A batch is split into groups of queries that share a database and a shape (d, n).
// Each group runs, per recursion level, one multi-task launch of the reply kernel (one
// task per query: its own query and output, and at levels >= 1 its own re-imported
// database), followed by one import launch that re-imports the level replies of all
// the group's queries together.  The arithmetic per query is exactly xpir_b200_reply's.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <mutex>
#include <vector>

#include "handles.h"
#include "kernels.h"
#include "params.h"
#include "xpir_b200.h"

using namespace xpir;

namespace {

int status_of(cudaError_t e) {
  if (e == cudaSuccess) return XPIR_B200_OK;
  (void)cudaGetLastError();
  if (e == cudaErrorMemoryAllocation) return XPIR_B200_ERR_NOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice) return XPIR_B200_ERR_NODEV;
  if (e == cudaErrorNotSupported) return XPIR_B200_ERR_ARG;
  return XPIR_B200_ERR_CUDA;
}

struct Shape {
  uint32_t d = 0;
  uint64_t P[XPIR_B200_MAX_LEVELS] = {};
  uint64_t groups[XPIR_B200_MAX_LEVELS] = {};
  uint64_t n_real0 = 0;
};

// Level shapes of a query against `db` (the level loop of generateReply(),
// pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:366-429).  False if invalid.
bool level_shapes(const xpir_b200_ctx *ctx, const xpir_b200_db *db, uint32_t d, const uint32_t *n, Shape *sh) {
  if (!db || db->ctx != ctx || d == 0 || d > XPIR_B200_MAX_LEVELS) return false;
  uint64_t slots = 1;
  for (uint32_t i = 0; i < d; i++) {
    if (n[i] == 0 || slots > UINT64_MAX / n[i]) return false;
    slots *= n[i];
  }
  if (slots < db->n_agg) return false;
  const uint64_t ct_bits = 2ull * 64 * ctx->ps.m * ctx->ps.N;
  sh->d = d;
  sh->n_real0 = db->n_agg;
  sh->P[0] = db->P;
  for (uint32_t lvl = 0; lvl < d; lvl++) {
    sh->groups[lvl] = 1;
    for (uint32_t j = lvl + 1; j < d; j++) sh->groups[lvl] *= n[j];
    if (lvl + 1 < d) sh->P[lvl + 1] = polys_for_bits(sh->P[lvl] * ct_bits, db->b, ctx->ps.N);
  }
  return true;
}

struct Group {
  const xpir_b200_db *db;
  uint32_t d;
  uint32_t n[XPIR_B200_MAX_LEVELS];
  Shape sh;
  std::vector<uint32_t> reqs;
};

struct Sizes {
  size_t ws_a = 0, ws_b = 0, tasks = 0;
};

Sizes sizes_of(const xpir_b200_ctx *ctx, const std::vector<Group> &groups) {
  const uint64_t mN = (uint64_t)ctx->ps.m * ctx->ps.N, ct_bytes = 2 * mN * 8;
  Sizes z;
  for (const Group &g : groups) {
    const uint64_t k = g.reqs.size();
    z.tasks += k * g.d;
    for (uint32_t lvl = 0; lvl + 1 < g.d; lvl++) {
      z.ws_a = std::max<size_t>(z.ws_a, k * g.sh.groups[lvl] * g.sh.P[lvl] * ct_bytes);
      z.ws_b = std::max<size_t>(z.ws_b, k * g.sh.groups[lvl] * g.sh.P[lvl + 1] * mN * 8);
    }
  }
  return z;
}

// Enqueues every launch of the batch on the context's stream.
cudaError_t enqueue(xpir_b200_ctx *ctx, const std::vector<Group> &groups, const xpir_b200_request *reqs,
                    uint64_t *ws_a, uint64_t *ws_b, ReplyTask *host_tasks, ReplyTask *dev_tasks) {
  const uint64_t mN = (uint64_t)ctx->ps.m * ctx->ps.N, ct_words = 2 * mN, ct_bytes = ct_words * 8;
  size_t task_off = 0;
  for (const Group &g : groups) {
    ParamSet ps = ctx->ps;
    ps.b = g.db->b;
    const DevModuli dm = make_dev_moduli(ps);
    const uint32_t k = (uint32_t)g.reqs.size();
    std::vector<const uint64_t *> db(k), q(k);
    std::vector<uint64_t *> out(k);
    uint64_t q_off = 0;
    for (uint32_t lvl = 0; lvl < g.d; lvl++) {
      const bool last = lvl + 1 == g.d;
      const uint64_t P = g.sh.P[lvl], groups_l = g.sh.groups[lvl];
      const uint64_t n_real = lvl == 0 ? g.sh.n_real0 : g.sh.groups[lvl - 1];
      for (uint32_t i = 0; i < k; i++) {
        const xpir_b200_request &r = reqs[g.reqs[i]];
        db[i] = lvl == 0 ? g.db->d_polys : ws_b + (uint64_t)i * n_real * P * mN;
        q[i] = (const uint64_t *)r.query + q_off;
        out[i] = last ? (uint64_t *)r.replies : ws_a + (uint64_t)i * groups_l * P * ct_words;
      }
      uint32_t launched = 0;
      cudaError_t e = launch_reply_tasks(db.data(), q.data(), out.data(), k, n_real, P, groups_l, g.n[lvl], ps, dm,
                                         host_tasks + task_off, dev_tasks + task_off, ctx->stream, &launched,
                                         ctx->status_dev, tuned_tile(ctx, P, g.n[lvl], groups_l), last);
      ctx->launches += launched;
      if (e != cudaSuccess) {
        fprintf(stderr, "xpir_b200: batched reply launch failed: %s (level %u of %u, P %llu, n_i %u, groups %llu, %u tasks)\n",
                cudaGetErrorName(e), lvl, g.d, (unsigned long long)P, g.n[lvl], (unsigned long long)groups_l, k);
        return e;
      }
      task_off += k;
      q_off += (uint64_t)g.n[lvl] * ct_words;
      if (last) break;
      // All queries' level replies are one run of k*groups elements of P ciphertexts; in
      // each query's row, groups past `active` replied exactly zero (and were not written).
      const AggSource as{(const uint8_t *)ws_a, (uint64_t)k * groups_l, P * ct_bytes, P * ct_bytes, 1};
      const ImportRows rows{k, groups_l, active_groups(n_real, g.n[lvl], groups_l)};
      launched = 0;
      e = launch_import(as, (uint64_t)k * groups_l, g.sh.P[lvl + 1], ps, dm, ctx->d_tables, ws_b, ctx->stream,
                        &rows, &launched);
      ctx->launches += launched;
      if (e != cudaSuccess) {
        fprintf(stderr, "xpir_b200: batched re-import launch failed: %s (level %u of %u, %u tasks)\n",
                cudaGetErrorName(e), lvl, g.d, k);
        return e;
      }
    }
  }
  return cudaSuccess;
}

}  // namespace

// A captured batch: its own workspaces and task tables, so that the graph stays valid
// whatever else the context does.
struct BatchPlan {
  std::vector<uint64_t> key;
  std::vector<uint64_t> db_ids;  // databases the graph reads
  uint64_t launches = 0;  // engine kernels in the captured graph
  void *ws_a = nullptr, *ws_b = nullptr, *dev_tasks = nullptr, *host_tasks = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~BatchPlan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaFree(ws_a);
    cudaFree(ws_b);
    cudaFree(dev_tasks);
    if (host_tasks) cudaFreeHost(host_tasks);
  }
};

namespace {

std::vector<uint64_t> plan_key(const xpir_b200_ctx *ctx, const xpir_b200_request *reqs, uint32_t count,
                               uint64_t tune_epoch) {
  std::vector<uint64_t> key{tune_epoch, (uint64_t)(uintptr_t)ctx, count};
  for (uint32_t i = 0; i < count; i++) {
    key.push_back(reqs[i].db ? reqs[i].db->id : 0);
    key.push_back(reqs[i].d);
    for (uint32_t j = 0; j < reqs[i].d && j < XPIR_B200_MAX_LEVELS; j++) key.push_back(reqs[i].n[j]);
    key.push_back((uint64_t)(uintptr_t)reqs[i].query);
    key.push_back((uint64_t)(uintptr_t)reqs[i].replies);
  }
  return key;
}

constexpr size_t kMaxPlans = 8;

}  // namespace

void xpir::drop_plans_of(xpir_b200_ctx *ctx, uint64_t db_id) {
  auto &plans = ctx->plans;
  plans.erase(std::remove_if(plans.begin(), plans.end(),
                             [db_id](const std::shared_ptr<BatchPlan> &pl) {
                               return std::find(pl->db_ids.begin(), pl->db_ids.end(), db_id) != pl->db_ids.end();
                             }),
              plans.end());
}

int xpir::reply_batch_impl(xpir_b200_ctx *ctx, xpir_b200_request *reqs, uint32_t count, int use_graph,
                           const WorkspaceFn *workspace) {
  if (!ctx || (!reqs && count)) return XPIR_B200_ERR_ARG;
  if (count == 0) return XPIR_B200_OK;
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return status_of(e);

  // Validate and group.
  const uint64_t ct_bytes = 2ull * ctx->ps.m * ctx->ps.N * 8;
  std::vector<Group> groups;
  int overall = XPIR_B200_OK;
  for (uint32_t i = 0; i < count; i++) {
    xpir_b200_request &r = reqs[i];
    r.nb_replies = 0;
    Shape sh;
    if (!r.query || !r.replies || !level_shapes(ctx, r.db, r.d, r.n, &sh) ||
        r.capacity_bytes < sh.P[sh.d - 1] * ct_bytes) {
      r.status = XPIR_B200_ERR_ARG;
      overall = XPIR_B200_ERR_ARG;
      continue;
    }
    r.status = XPIR_B200_OK;
    auto it = std::find_if(groups.begin(), groups.end(), [&](const Group &g) {
      return g.db == r.db && g.d == r.d && memcmp(g.n, r.n, r.d * sizeof(uint32_t)) == 0;
    });
    if (it == groups.end()) {
      Group g;
      g.db = r.db;
      g.d = r.d;
      memset(g.n, 0, sizeof(g.n));
      memcpy(g.n, r.n, r.d * sizeof(uint32_t));
      g.sh = sh;
      groups.push_back(g);
      it = groups.end() - 1;
    }
    it->reqs.push_back(i);
  }
  if (groups.empty()) return overall;
  const Sizes z = sizes_of(ctx, groups);
  *ctx->status_host = 0;

  auto finish = [&](cudaError_t err) -> int {
    const cudaError_t se = cudaStreamSynchronize(ctx->stream);  // also on error: nothing left in flight
    if (err == cudaSuccess) err = se;
    if (err != cudaSuccess) ctx->last_error = err;
    int rc = status_of(err);
    if (rc == XPIR_B200_OK && *(volatile int *)ctx->status_host != 0) rc = XPIR_B200_ERR_TIMEOUT;
    for (const Group &g : groups)
      for (uint32_t i : g.reqs) {
        reqs[i].status = rc;
        if (rc == XPIR_B200_OK) reqs[i].nb_replies = g.sh.P[g.d - 1];
      }
    return rc != XPIR_B200_OK ? rc : overall;
  };

  if (!use_graph) {
    // Workspaces from the caller, or the context's own, grown on demand and kept; the
    // task table likewise.  After the first calls an uncaptured batch allocates and frees
    // nothing, so it never synchronises the device (other contexts' streams keep running).
    void *wa = nullptr, *wb = nullptr;
    if (workspace) {
      if ((e = (*workspace)(z.ws_a, z.ws_b, &wa, &wb)) != cudaSuccess) return finish(e);
    } else {
      if (z.ws_a > ctx->ws_a_bytes) {
        cudaFree(ctx->ws_a);
        ctx->ws_a = nullptr;
        ctx->ws_a_bytes = 0;
        if ((e = cudaMalloc(&ctx->ws_a, z.ws_a)) != cudaSuccess) return finish(e);
        ctx->ws_a_bytes = z.ws_a;
      }
      if (z.ws_b > ctx->ws_b_bytes) {
        cudaFree(ctx->ws_b);
        ctx->ws_b = nullptr;
        ctx->ws_b_bytes = 0;
        if ((e = cudaMalloc(&ctx->ws_b, z.ws_b)) != cudaSuccess) return finish(e);
        ctx->ws_b_bytes = z.ws_b;
      }
      wa = ctx->ws_a;
      wb = ctx->ws_b;
    }
    if (z.tasks > ctx->tasks_cap) {
      cudaFree(ctx->tasks_dev);
      if (ctx->tasks_host) cudaFreeHost(ctx->tasks_host);
      ctx->tasks_dev = ctx->tasks_host = nullptr;
      ctx->tasks_cap = 0;
      const size_t cap = std::max<size_t>(z.tasks, 64);
      e = cudaMalloc(&ctx->tasks_dev, cap * sizeof(ReplyTask));
      if (e == cudaSuccess) e = cudaMallocHost(&ctx->tasks_host, cap * sizeof(ReplyTask));
      if (e != cudaSuccess) return finish(e);
      ctx->tasks_cap = cap;
    }
    // The pinned table may be rewritten here: the previous call on this context ended
    // with a stream synchronisation, so its copy has completed.
    e = enqueue(ctx, groups, reqs, (uint64_t *)wa, (uint64_t *)wb, (ReplyTask *)ctx->tasks_host,
                (ReplyTask *)ctx->tasks_dev);
    return finish(e);
  }

  // Graph path: replay a captured plan for the same request list, or capture one.
  const std::vector<uint64_t> key = plan_key(ctx, reqs, count, ctx->tune_epoch);
  for (auto &pl : ctx->plans)
    if (pl->key == key) {
      ctx->launches += pl->launches;
      return finish(cudaGraphLaunch(pl->exec, ctx->stream));
    }
  auto plan = std::make_shared<BatchPlan>();
  plan->key = key;
  for (const Group &g : groups) plan->db_ids.push_back(g.db->id);
  e = cudaMalloc(&plan->ws_a, std::max<size_t>(z.ws_a, 256));
  if (e == cudaSuccess) e = cudaMalloc(&plan->ws_b, std::max<size_t>(z.ws_b, 256));
  if (e == cudaSuccess) e = cudaMalloc(&plan->dev_tasks, z.tasks * sizeof(ReplyTask));
  if (e == cudaSuccess) e = cudaMallocHost(&plan->host_tasks, z.tasks * sizeof(ReplyTask));
  // One eager run first: it sets the kernels' attributes outside the capture and
  // produces this submission's replies.
  if (e == cudaSuccess)
    e = enqueue(ctx, groups, reqs, (uint64_t *)plan->ws_a, (uint64_t *)plan->ws_b, (ReplyTask *)plan->host_tasks,
                (ReplyTask *)plan->dev_tasks);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    const uint64_t before = ctx->launches;
    const cudaError_t ee = enqueue(ctx, groups, reqs, (uint64_t *)plan->ws_a, (uint64_t *)plan->ws_b,
                                   (ReplyTask *)plan->host_tasks, (ReplyTask *)plan->dev_tasks);
    plan->launches = ctx->launches - before;
    ctx->launches = before;  // captured, not launched
    e = cudaStreamEndCapture(ctx->stream, &plan->graph);
    if (ee != cudaSuccess) e = ee;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&plan->exec, plan->graph, 0);
  if (e != cudaSuccess) return finish(e);
  if (ctx->plans.size() >= kMaxPlans) ctx->plans.erase(ctx->plans.begin());
  ctx->plans.push_back(plan);
  return finish(cudaSuccess);
}

extern "C" int xpir_b200_reply_batch(xpir_b200_ctx *ctx, xpir_b200_request *reqs, uint32_t count, int use_graph) {
  return reply_batch_impl(ctx, reqs, count, use_graph, nullptr);
}

extern "C" int xpir_b200_autotune(xpir_b200_ctx *ctx, const xpir_b200_db *db, uint32_t d, const uint32_t *n,
                                  const void *query_dev, int *tile0) {
  if (!ctx || !n || !query_dev) return XPIR_B200_ERR_ARG;
  Shape sh;
  if (!level_shapes(ctx, db, d, n, &sh)) return XPIR_B200_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return status_of(e);
  ParamSet ps = ctx->ps;
  ps.b = db->b;
  const DevModuli dm = make_dev_moduli(ps);
  const uint64_t mN = (uint64_t)ps.m * ps.N, ct_words = 2 * mN, ct_bytes = ct_words * 8;
  size_t rep_max = 0, next_max = 0;
  for (uint32_t lvl = 0; lvl < d; lvl++) {
    rep_max = std::max<size_t>(rep_max, sh.groups[lvl] * sh.P[lvl] * ct_bytes);
    if (lvl + 1 < d) next_max = std::max<size_t>(next_max, sh.groups[lvl] * sh.P[lvl + 1] * mN * 8);
  }
  uint64_t *rep = nullptr, *next = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  e = cudaMalloc(&rep, rep_max);
  if (e == cudaSuccess && next_max) e = cudaMalloc(&next, next_max);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  *ctx->status_host = 0;
  const uint64_t *in = db->d_polys;
  const uint64_t *q = (const uint64_t *)query_dev;
  uint64_t in_real = db->n_agg;
  for (uint32_t lvl = 0; lvl < d && e == cudaSuccess; lvl++) {
    ReplyLevelArgs a{in, in_real, sh.P[lvl], sh.groups[lvl], n[lvl], q, rep};
    int best = -1;
    float best_ms = 0;
    for (int cand : tile_candidates(sh.P[lvl])) {
      float ms = 0;
      for (int rep_i = 0; rep_i < 2 && e == cudaSuccess; rep_i++) {  // the first run warms up
        e = cudaEventRecord(e0, ctx->stream);
        if (e == cudaSuccess) e = launch_reply_level(a, ps, dm, ctx->stream, nullptr, ctx->status_dev, cand);
        if (e == cudaSuccess) e = cudaEventRecord(e1, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      }
      if (e != cudaSuccess) break;
      if (best < 0 || ms < best_ms) {
        best = cand;
        best_ms = ms;
      }
    }
    if (e != cudaSuccess) break;
    ctx->tuned[std::make_tuple(sh.P[lvl], (uint64_t)n[lvl], sh.groups[lvl])] = best;
    if (lvl == 0 && tile0) *tile0 = best;
    q += (uint64_t)n[lvl] * ct_words;
    if (lvl + 1 == d) break;
    const AggSource as{(const uint8_t *)rep, sh.groups[lvl], sh.P[lvl] * ct_bytes, sh.P[lvl] * ct_bytes, 1};
    e = launch_import(as, sh.groups[lvl], sh.P[lvl + 1], ps, dm, ctx->d_tables, next, ctx->stream);
    in = next;
    in_real = sh.groups[lvl];
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  ctx->tune_epoch++;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(rep);
  cudaFree(next);
  if (e == cudaSuccess && *(volatile int *)ctx->status_host != 0) return XPIR_B200_ERR_TIMEOUT;
  return status_of(e);
}

extern "C" int xpir_b200_set_level_tile(xpir_b200_ctx *ctx, uint64_t P, uint32_t n_i, uint64_t groups, int tile) {
  if (!ctx || P == 0 || n_i == 0 || groups == 0) return XPIR_B200_ERR_ARG;
  if (tile != -1 && !tile_fits(tile, P)) return XPIR_B200_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  const auto key = std::make_tuple(P, (uint64_t)n_i, groups);
  if (tile == -1)
    ctx->tuned.erase(key);
  else
    ctx->tuned[key] = tile;
  ctx->tune_epoch++;
  return XPIR_B200_OK;
}

extern "C" int xpir_b200_tile_count(void) { return tile_count(); }

// The optimizer's per-plaintext costs (pir/replyGenerator/PIROptimizer.cpp:155-209): a
// one-dimensional query over n[0] = 4 elements of `plaintexts` polys each, doubled until
// one reply takes `target_s` or the database reaches 2^30 ciphertext bits (the reference's
// limit), then reply time and import time divided by the plaintexts in the database.
extern "C" int xpir_b200_measure_costs(xpir_b200_ctx *ctx, uint32_t security_bits, double target_s,
                                       double *reply_s_per_plaintext, double *import_s_per_plaintext) {
  if (!ctx || !reply_s_per_plaintext || !import_s_per_plaintext || security_bits == 0) return XPIR_B200_ERR_ARG;
  const uint32_t N = ctx->ps.N, m = ctx->ps.m, n0 = 4;
  const int32_t b = xpir_b200_bits_per_coeff(N, m, security_bits, n0);
  if (b <= 0) return XPIR_B200_ERR_ARG;
  const uint64_t ct_bits = 2ull * 64 * m * N, abs_bytes = (uint64_t)b * N / 8;
  if (target_s <= 0) target_s = 0.05;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return status_of(e);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e != cudaSuccess) return status_of(e);
  int rc = XPIR_B200_OK;
  double reply_s = 0, import_s = 0;
  uint64_t plaintexts = 4, used = 4;
  std::vector<uint8_t> bytes;
  std::vector<uint64_t> query((uint64_t)n0 * 2 * m * N, 1), replies;
  for (;;) {
    const uint64_t L = plaintexts * abs_bytes;
    bytes.assign((uint64_t)n0 * L, 0x5a);
    float ms_import = 0, ms_reply = 0;
    xpir_b200_db *db = nullptr;
    e = cudaEventRecord(e0, ctx->stream);
    if (e == cudaSuccess) rc = xpir_b200_db_import(ctx, bytes.data(), n0, L, L, 1, (uint32_t)b, 0, &db);
    if (e == cudaSuccess && rc == XPIR_B200_OK) e = cudaEventRecord(e1, ctx->stream);
    if (e == cudaSuccess && rc == XPIR_B200_OK) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess && rc == XPIR_B200_OK) e = cudaEventElapsedTime(&ms_import, e0, e1);
    if (e == cudaSuccess && rc == XPIR_B200_OK) {
      uint64_t P = 0, nagg = 0, dev = 0;
      uint32_t bb = 0;
      xpir_b200_db_info(db, &nagg, &P, &bb, &dev);
      replies.assign(P * 2 * m * N, 0);
      void *dq = nullptr, *dr = nullptr;
      e = cudaMalloc(&dq, query.size() * 8);
      if (e == cudaSuccess) e = cudaMalloc(&dr, replies.size() * 8);
      if (e == cudaSuccess) e = cudaMemcpy(dq, query.data(), query.size() * 8, cudaMemcpyHostToDevice);
      uint64_t cnt = 0;
      for (int rep = 0; rep < 3 && e == cudaSuccess && rc == XPIR_B200_OK; rep++) {  // warm-up, then timed
        if (rep == 2) e = cudaEventRecord(e0, ctx->stream);
        rc = xpir_b200_reply(ctx, db, 1, &n0, dq, 1, dr, replies.size() * 8, 1, &cnt);
        if (rep == 2 && e == cudaSuccess) e = cudaEventRecord(e1, ctx->stream);
      }
      if (e == cudaSuccess && rc == XPIR_B200_OK) e = cudaEventSynchronize(e1);
      if (e == cudaSuccess && rc == XPIR_B200_OK) e = cudaEventElapsedTime(&ms_reply, e0, e1);
      cudaFree(dq);
      cudaFree(dr);
    }
    if (db) xpir_b200_db_free(db);
    if (e != cudaSuccess || rc != XPIR_B200_OK) break;
    reply_s = ms_reply / 1e3;
    import_s = ms_import / 1e3;
    used = plaintexts;
    if (reply_s >= target_s || plaintexts * 2 * n0 * ct_bits >= (1ull << 30)) break;
    plaintexts *= 2;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return status_of(e);
  if (rc != XPIR_B200_OK) return rc;
  *reply_s_per_plaintext = reply_s / ((double)n0 * used);
  *import_s_per_plaintext = import_s / ((double)n0 * used);
  return XPIR_B200_OK;
}
