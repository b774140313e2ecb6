// xpir_b200_reply_noalloc: the reply of one device-resident query with no device or
// host allocation in the call.  For callers that cannot allocate while they serve a
// request (memory set up in advance under a fixed budget, or code running inside an
// allocator hook); see include/xpir_b200.h.
//
// The intermediate data of a recursive query lives in one file-scope device array of
// XPIR_B200_NOALLOC_SCRATCH_BYTES: level replies at its start, the next level's
// database after them.  Host code cannot use the array's name as a device address, so
// xpir_b200_ctx_create looks the address up on its device with cudaGetSymbolAddress
// (which, under lazy module loading, is also when this module and its array are placed
// on the device) and caches it per device.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "handles.h"
#include "kernels.h"
#include "params.h"
#include "xpir_b200.h"

namespace {

// Every GPU that loads the library holds this until the process exits.
static __device__ __align__(256) uint8_t g_reply_scratch[XPIR_B200_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of g_reply_scratch on `device` (which must be current); looked up once
// per device.
cudaError_t scratch_address(int device, uint8_t **out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_reply_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = p;
  }
  *out = (uint8_t *)g_scratch_addr[device];
  return cudaSuccess;
}

int status_of(cudaError_t e) {
  if (e == cudaSuccess) return XPIR_B200_OK;
  (void)cudaGetLastError();
  if (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice) return XPIR_B200_ERR_NODEV;
  if (e == cudaErrorNotSupported || e == cudaErrorInvalidValue) return XPIR_B200_ERR_ARG;
  return XPIR_B200_ERR_CUDA;
}

uint64_t round_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

bool mul_ok(uint64_t a, uint64_t b, uint64_t *out) {
  if (a != 0 && b > UINT64_MAX / a) return false;
  *out = a * b;
  return true;
}

// Restores the caller's current device when the call returns.
struct DeviceRestore {
  int saved = -1;
  DeviceRestore() {
    if (cudaGetDevice(&saved) != cudaSuccess) {
      (void)cudaGetLastError();
      saved = -1;
    }
  }
  ~DeviceRestore() {
    if (saved >= 0) cudaSetDevice(saved);
  }
};

}  // namespace

cudaError_t xpir::prepare_noalloc_scratch(int device) {
  uint8_t *p = nullptr;
  return scratch_address(device, &p);
}

extern "C" int xpir_b200_reply_noalloc(xpir_b200_ctx *ctx, const xpir_b200_db *db, uint32_t d, const uint32_t *n,
                                       const void *query_dev, void *replies_dev, uint64_t capacity_bytes,
                                       uint64_t *nb_replies) {
  using namespace xpir;
  if (!ctx || !db || !n || !query_dev || !replies_dev || d == 0 || d > XPIR_B200_MAX_LEVELS) return XPIR_B200_ERR_ARG;
  if (db->ctx != ctx) return XPIR_B200_ERR_ARG;
  uint64_t slots = 1;
  for (uint32_t i = 0; i < d; i++) {
    if (n[i] == 0 || slots > UINT64_MAX / n[i]) return XPIR_B200_ERR_ARG;
    slots *= n[i];
  }
  if (slots < db->n_agg) return XPIR_B200_ERR_ARG;

  ParamSet ps = ctx->ps;
  ps.b = db->b;
  const DevModuli dm = make_dev_moduli(ps);
  const uint64_t mN = (uint64_t)ps.m * ps.N, ct_words = 2 * mN, ct_bytes = ct_words * 8;

  // Shapes of every level, and the scratch they need: level replies (all levels but
  // the last) at offset 0, the next level's database after them.  Every product is
  // checked, so that no wrapped size can pass the scratch limit.
  uint64_t Ps[XPIR_B200_MAX_LEVELS], groups[XPIR_B200_MAX_LEVELS];
  uint64_t need_a = 0, need_b = 0;
  Ps[0] = db->P;
  for (uint32_t lvl = 0; lvl < d; lvl++) {
    groups[lvl] = 1;
    for (uint32_t j = lvl + 1; j < d; j++) groups[lvl] *= n[j];  // <= prod(n), checked above
    if (lvl + 1 < d) {
      uint64_t gp, rep_bytes, bits, next_polys, next_bytes;
      if (!mul_ok(groups[lvl], Ps[lvl], &gp) || !mul_ok(gp, ct_bytes, &rep_bytes)) return XPIR_B200_ERR_ARG;
      if (!mul_ok(Ps[lvl], ct_bytes * 8, &bits)) return XPIR_B200_ERR_ARG;
      Ps[lvl + 1] = polys_for_bits(bits, ps.b, ps.N);
      if (!mul_ok(groups[lvl], Ps[lvl + 1], &next_polys) || !mul_ok(next_polys, mN * 8, &next_bytes))
        return XPIR_B200_ERR_ARG;
      if (rep_bytes > need_a) need_a = rep_bytes;
      if (next_bytes > need_b) need_b = next_bytes;
    }
  }
  // Each size alone must fit; then the sum below cannot wrap.
  if (need_a > XPIR_B200_NOALLOC_SCRATCH_BYTES || need_b > XPIR_B200_NOALLOC_SCRATCH_BYTES)
    return XPIR_B200_ERR_ARG;
  const uint64_t off_b = round_up(need_a, 256);
  if (off_b + need_b > XPIR_B200_NOALLOC_SCRATCH_BYTES) return XPIR_B200_ERR_ARG;  // does not fit the scratch
  const uint64_t final_count = Ps[d - 1];
  uint64_t final_bytes;
  if (!mul_ok(final_count, ct_bytes, &final_bytes) || capacity_bytes < final_bytes) return XPIR_B200_ERR_ARG;

  std::lock_guard<std::mutex> lock(ctx->mu);
  DeviceRestore restore;
  cudaError_t e = cudaSetDevice(ctx->device);
  uint8_t *scratch = nullptr;
  if (e == cudaSuccess && d > 1) e = scratch_address(ctx->device, &scratch);
  if (e != cudaSuccess) return status_of(e);

  *ctx->status_host = 0;
  const uint64_t *in = db->d_polys;
  const uint64_t *q = (const uint64_t *)query_dev;
  uint64_t in_real = db->n_agg;
  for (uint32_t lvl = 0; lvl < d; lvl++) {
    const bool last = lvl + 1 == d;
    uint64_t *rep = last ? (uint64_t *)replies_dev : (uint64_t *)scratch;
    uint32_t launched = 0;
    // As xpir_b200_reply: intermediate levels leave the replies of groups without data
    // unwritten, and the next import fills those groups with their constant poly.
    ReplyLevelArgs a{in, in_real, Ps[lvl], groups[lvl], n[lvl], q, rep};
    a.write_idle = last;
    const uint64_t active = active_groups(in_real, n[lvl], groups[lvl]);
    e = launch_reply_level(a, ps, dm, ctx->stream, &launched, ctx->status_dev,
                           tuned_tile(ctx, Ps[lvl], n[lvl], groups[lvl]));
    ctx->launches += launched;
    if (e != cudaSuccess) return status_of(e);
    q += (uint64_t)n[lvl] * ct_words;
    if (last) break;
    uint64_t *next = (uint64_t *)(scratch + off_b);
    const AggSource as{(const uint8_t *)rep, groups[lvl], Ps[lvl] * ct_bytes, Ps[lvl] * ct_bytes, 1};
    const ImportRows rows{1, groups[lvl], active};
    launched = 0;
    e = launch_import(as, groups[lvl], Ps[lvl + 1], ps, dm, ctx->d_tables, next, ctx->stream, &rows, &launched);
    ctx->launches += launched;
    if (e != cudaSuccess) return status_of(e);
    in = next;
    in_real = groups[lvl];
  }
  e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return status_of(e);
  if (*(volatile int *)ctx->status_host != 0) return XPIR_B200_ERR_TIMEOUT;
  if (nb_replies) *nb_replies = final_count;
  return XPIR_B200_OK;
}
