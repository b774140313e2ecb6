// Client-side reply extraction on the GPU: NFLLWE decryption of every reply ciphertext
// and the recursion back to the element (crypto/NFLLWE.cpp:375-475, 515-551;
// pir/replyExtraction/PIRReplyExtraction_internal.cpp:41-106).
//
// Per level, two kernels:
//   decrypt_poly_kernel  one CTA per (ciphertext, modulus): m = b - a*s (lazy Shoup MAC
//                        then submod, crypto/NFLlib.hpp:255-267, 303-321), bit reversal,
//                        the lazy NTT with the inverse twiddles, bit reversal back, and
//                        the N^-1 phi^-i scaling (crypto/NFLlib.hpp:548-566, 613-626);
//   lift_pack_kernel     one thread per (ciphertext, coefficient): the CRT lift to
//                        [0, P) by mixed radix (the unique value NFLlib::poly2mpz also
//                        computes, crypto/NFLlib.cpp:504-532), centred (x - P when
//                        2x > P), its low b bits appended LSB-first to the ciphertext's
//                        plaintext bytes (the bit order of NFLlib::serializeData32/64,
//                        crypto/NFLlib.cpp:412-495).
// The level's plaintext bytes are the next level's ciphertexts; the innermost level's
// are the aggregated element.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "handles.h"
#include "kernels.h"
#include "modarith.cuh"
#include "ntt.cuh"
#include "params.h"
#include "xpir_b200.h"

namespace xpir {
namespace {

constexpr uint32_t kMaxLiftModuli = 4;  // b < 128 bits per coefficient
constexpr int kLimbs = kMaxLiftModuli + 1;

// Mixed-radix constants: x = v0 + v1*M1 + ... with M_c = p_0*...*p_{c-1}.
struct LiftConsts {
  uint64_t P[kLimbs];              // product of the moduli
  uint64_t M[kMaxLiftModuli][kLimbs];
  uint64_t inv[kMaxLiftModuli];    // M_c^-1 mod p_c
  uint64_t inv_shoup[kMaxLiftModuli];  // floor(inv * 2^64 / p_c)
};

// Exact reductions modulo one of XPIR's moduli (2^60 < p < 2^61 with D = 2^61 - p below
// 2^23 for all 17 of them), which give the unique residue the reference's GMP lift
// computes.  A 64-bit word w: q0 = w >> 61 <= 7 and w - q0*p = (w mod 2^61) + q0*D lies
// in [0, 2p) whenever 9*D < 2^61.
__device__ __forceinline__ uint64_t mod_word(uint64_t w, uint64_t p, uint64_t np) {
  const uint64_t r = w + (w >> 61) * np;
  return r >= p ? r - p : r;
}

// h*2^64 + l mod p for h < p: h*2^64 mod p = h*2^64 - f*p with f = floor(h*2^64/p) (the
// Shoup factor of h), whose low word is f*(2^64 - p).
__device__ __forceinline__ uint64_t mod_two_words(uint64_t h, uint64_t l, uint64_t p, uint64_t np, uint32_t delta) {
  const uint64_t s = shoup_factor8_np(h, p, np, delta) * np + mod_word(l, p, np);  // < 2p
  return s >= p ? s - p : s;
}

// x (its low nl of kLimbs little-endian limbs) mod p, from the top limb down; the loop is
// unrolled over all limbs so that x stays in registers.
__device__ __forceinline__ uint64_t limbs_mod_fast(const uint64_t (&x)[kLimbs], int nl, uint64_t p, uint64_t np,
                                                   uint32_t delta) {
  uint64_t r = 0;
#pragma unroll
  for (int l = kLimbs - 1; l >= 0; l--) {
    if (l == nl - 1) r = mod_word(x[l], p, np);
    else if (l < nl - 1) r = mod_two_words(r, x[l], p, np, delta);
  }
  return r;
}

__global__ void __launch_bounds__(256, 4) decrypt_poly_kernel(const uint64_t *__restrict__ ct,
                                                           const uint64_t *__restrict__ sk,
                                                           const uint64_t *__restrict__ sks,
                                                           const uint64_t *__restrict__ tables, uint32_t N,
                                                           uint32_t log_n, uint32_t m, const DevModuli dm,
                                                           uint64_t *__restrict__ res) {
  extern __shared__ uint64_t poly[];
  const uint32_t c = blockIdx.y;
  const uint64_t j = blockIdx.x;
  const uint64_t p = dm.p[c];
  const uint64_t *a = ct + (j * 2 * m + c) * N, *b = ct + (j * 2 * m + m + c) * N;
  const uint64_t *s = sk + (uint64_t)c * N, *ss = sks + (uint64_t)c * N;
  const uint32_t shift = 32 - log_n;
#pragma unroll 4
  for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {  // unrolled: several rows of loads in flight
    const uint64_t temp = shoup_mac(0, a[i], s[i], ss[i], p);  // in [0, p)
    const uint64_t y = (temp < p) ? p - temp : p - temp % p;
    uint64_t z = b[i] + y;
    z -= (z >= p) ? p : 0;
    poly[swz(__brev(i) >> shift)] = z;
  }
  __syncthreads();
  const uint64_t *tab = tables + (uint64_t)c * kTableSlots * N;
  ntt_lazy_rb<3>(poly, tab + kInvOmega * N, tab + kInvOmegaShoup * N, N, log_n, p,
                 [&](uint32_t k) { return poly[swz(k)]; });
  const uint64_t *iphi = tab + kInvPhi * N, *iphis = tab + kInvPhiShoup * N;
  uint64_t *o = res + (j * m + c) * N;
  // In output order (coalesced global loads and stores); the bit reversal is its own
  // inverse, so output k reads transform slot brev(k).
  for (uint32_t k = threadIdx.x; k < N; k += blockDim.x)
    o[k] = shoup_mul(poly[swz(__brev(k) >> shift)], iphi[k], iphis[k], p);
}

__global__ void __launch_bounds__(256) lift_pack_kernel(const uint64_t *__restrict__ res, uint64_t nct, uint32_t N,
                                                        uint32_t m, uint32_t bits, const LiftConsts lc,
                                                        const DevModuli dm, unsigned long long *__restrict__ out) {
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (t >= nct * N) return;
  const uint64_t j = t / N, i = t % N;
  uint64_t x[kLimbs] = {};
#pragma unroll
  for (uint32_t c = 0; c < kMaxLiftModuli; c++) {  // unrolled: static indexes into x and the constants
    if (c >= m) break;
    const uint64_t p = dm.p[c], np = 0 - p;
    const uint32_t delta = (uint32_t)dm.shoup_delta[c];
    const uint64_t r = mod_word(res[(j * m + c) * N + i], p, np);
    // x < p_0*...*p_{c-1} < 2^(61c): ceil(61c/64) limbs
    const uint64_t have = c ? limbs_mod_fast(x, (int)((61 * c + 63) / 64), p, np, delta) : 0;
    uint64_t t = r + p - have;
    t = t >= p ? t - p : t;
    const uint64_t v = c ? shoup_mul(t, lc.inv[c], lc.inv_shoup[c], p) : r;
    unsigned __int128 carry = 0;  // x += M_c * v
#pragma unroll
    for (int l = 0; l < kLimbs; l++) {
      const unsigned __int128 s = (unsigned __int128)lc.M[c][l] * v + x[l] + carry;
      x[l] = (uint64_t)s;
      carry = s >> 64;
    }
  }
  // centred: x - P when 2x > P
  int cmp = 0;  // sign of 2x - P (x < P < 2^244: 2x fits the limbs)
#pragma unroll
  for (int l = kLimbs - 1; l >= 0; l--) {  // unrolled (static limb indexes: registers)
    const uint64_t x2 = (x[l] << 1) | (l ? x[l - 1] >> 63 : 0);
    if (cmp == 0 && x2 != lc.P[l]) cmp = x2 > lc.P[l] ? 1 : -1;
  }
  unsigned __int128 v = ((unsigned __int128)x[1] << 64) | x[0];
  if (cmp > 0) v -= ((unsigned __int128)lc.P[1] << 64) | lc.P[0];
  if (bits < 128) v &= (((unsigned __int128)1) << bits) - 1;
  // append at bit offset i*bits of ciphertext j's plaintext (bits*N/64 words per ciphertext)
  const uint64_t pos = (uint64_t)i * bits, words = (uint64_t)bits * N / 64;
  unsigned long long *w = out + j * words + (pos >> 6);
  const uint32_t sh = (uint32_t)(pos & 63);
  const unsigned __int128 lo = v << sh;  // bits [sh, sh+bits) of a 192-bit window
  const uint64_t w0 = (uint64_t)lo, w1 = (uint64_t)(lo >> 64);
  const uint64_t w2 = sh ? (uint64_t)(v >> (128 - sh)) : 0;
  if (w0) atomicOr(w, (unsigned long long)w0);
  if (w1) atomicOr(w + 1, (unsigned long long)w1);
  if (w2) atomicOr(w + 2, (unsigned long long)w2);
}

// Limb helpers on the host.
void limbs_mul_small(uint64_t *M, uint64_t v) {
  unsigned __int128 carry = 0;
  for (int i = 0; i < kLimbs; i++) {
    const unsigned __int128 t = (unsigned __int128)M[i] * v + carry;
    M[i] = (uint64_t)t;
    carry = t >> 64;
  }
}

uint64_t limbs_mod_host(const uint64_t *x, uint64_t p) {
  unsigned __int128 r = 0;
  for (int i = kLimbs - 1; i >= 0; i--) r = ((r << 64) | x[i]) % p;
  return (uint64_t)r;
}

uint64_t powmod_host(uint64_t a, uint64_t e, uint64_t p) {
  uint64_t r = 1;
  a %= p;
  while (e) {
    if (e & 1) r = (uint64_t)(((unsigned __int128)r * a) % p);
    a = (uint64_t)(((unsigned __int128)a * a) % p);
    e >>= 1;
  }
  return r;
}

// Ciphertexts decrypted at level lvl: PIRReplyExtraction_internal::extractReply's float
// arithmetic (…_internal.cpp:50-58).
uint64_t extract_count(uint64_t agg_bytes, uint32_t lvl, uint32_t bits, uint32_t N, uint32_t m) {
  const float abs_bytes = (float)((uint64_t)bits * N / 8), ct_bytes = (float)(16ull * m * N);
  uint64_t nbr = (uint64_t)std::ceil((float)agg_bytes / abs_bytes);
  for (uint32_t i = 1; i < lvl; i++) {
    const float t = (float)nbr * ct_bytes;
    nbr = (uint64_t)std::ceil(t / abs_bytes);
  }
  return nbr;
}

int status_of(cudaError_t e) {
  if (e == cudaSuccess) return XPIR_B200_OK;
  (void)cudaGetLastError();
  if (e == cudaErrorMemoryAllocation) return XPIR_B200_ERR_NOMEM;
  return XPIR_B200_ERR_CUDA;
}

}  // namespace
}  // namespace xpir

using namespace xpir;

extern "C" uint64_t xpir_b200_extract_count(uint64_t aggregated_bytes, uint32_t level, uint32_t bits_per_coeff,
                                            uint32_t poly_degree, uint32_t nb_moduli) {
  if (level == 0 || bits_per_coeff == 0 || poly_degree == 0 || nb_moduli == 0) return 0;
  return extract_count(aggregated_bytes, level, bits_per_coeff, poly_degree, nb_moduli);
}

extern "C" int xpir_b200_extract(xpir_b200_ctx *ctx, const uint64_t *secret_key, uint32_t d, uint32_t bits_per_coeff,
                                 uint64_t aggregated_bytes, const void *replies, uint64_t nb_replies,
                                 int replies_on_device, void *plaintext, uint64_t capacity_bytes, int out_on_device) {
  if (!ctx || !secret_key || !replies || !plaintext || d == 0 || d > XPIR_B200_MAX_LEVELS || aggregated_bytes == 0)
    return XPIR_B200_ERR_ARG;
  const ParamSet &ps = ctx->ps;
  const uint32_t N = ps.N, m = ps.m, bits = bits_per_coeff;
  if (m > kMaxLiftModuli || bits == 0 || bits >= 128 || bits >= 61 * m || (uint64_t)bits * N % 64 != 0)
    return XPIR_B200_ERR_ARG;
  if (capacity_bytes < aggregated_bytes) return XPIR_B200_ERR_ARG;
  for (uint32_t c = 0; c < m; c++) {  // the lift's reductions (mod_word, mod_two_words) assume these
    const uint64_t p = ps.mod[c].p;
    if (p <= (1ull << 60) || p >= (1ull << 61) || (1ull << 61) - p >= (1ull << 57) || !shoup_factor_ok(p))
      return XPIR_B200_ERR_ARG;
  }
  const uint64_t top = extract_count(aggregated_bytes, d, bits, N, m);
  if (nb_replies < top) return XPIR_B200_ERR_ARG;
  const uint64_t mN = (uint64_t)m * N, ct_words = 2 * mN, abs_words = (uint64_t)bits * N / 64;

  // Host constants of the mixed-radix lift (the key's Shoup factors are computed on the device).
  LiftConsts lc;
  memset(&lc, 0, sizeof(lc));
  lc.P[0] = 1;
  for (uint32_t c = 0; c < m; c++) {
    const uint64_t p = ps.mod[c].p;
    memcpy(lc.M[c], lc.P, sizeof(lc.P));
    lc.inv[c] = c ? powmod_host(limbs_mod_host(lc.P, p), p - 2, p) : 1;
    lc.inv_shoup[c] = (uint64_t)(((unsigned __int128)lc.inv[c] << 64) / p);
    limbs_mul_small(lc.P, p);
  }
  const DevModuli dm = make_dev_moduli(ps);

  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return status_of(e);
  cudaStream_t st = ctx->stream;
  uint64_t *d_sk = nullptr, *d_sks = nullptr, *d_in = nullptr, *d_res = nullptr, *d_out = nullptr;
  auto cleanup = [&]() {
    cudaFreeAsync(d_sk, st);
    cudaFreeAsync(d_sks, st);
    cudaFreeAsync(d_in, st);
    cudaFreeAsync(d_res, st);
    cudaFreeAsync(d_out, st);
  };
  e = cudaMallocFromPoolAsync((void **)&d_sk, mN * 8, ctx->pool, st);
  if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void **)&d_sks, mN * 8, ctx->pool, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_sk, secret_key, mN * 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    e = launch_key_shoup(d_sk, d_sks, N, m, dm, st);
    ctx->launches++;
  }
  const uint64_t *level_in = (const uint64_t *)replies;
  if (e == cudaSuccess && !replies_on_device) {
    e = cudaMallocFromPoolAsync((void **)&d_in, top * ct_words * 8, ctx->pool, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_in, replies, top * ct_words * 8, cudaMemcpyHostToDevice, st);
    level_in = d_in;
  }
  if (e == cudaSuccess) e = allow_max_dynamic_smem((const void *)decrypt_poly_kernel);
  for (uint32_t lvl = d; lvl >= 1 && e == cudaSuccess; lvl--) {
    const uint64_t nbr = extract_count(aggregated_bytes, lvl, bits, N, m);
    uint64_t *res = nullptr, *out = nullptr;
    // The plaintext (plus slack for the last value's straddling word) is read by the
    // next level as its ciphertexts: size it for both.
    uint64_t out_words = nbr * abs_words + 3;
    if (lvl > 1) out_words = std::max<uint64_t>(out_words, extract_count(aggregated_bytes, lvl - 1, bits, N, m) * ct_words);
    e = cudaMallocFromPoolAsync((void **)&res, nbr * mN * 8, ctx->pool, st);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void **)&out, out_words * 8, ctx->pool, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(out, 0, out_words * 8, st);
    if (e == cudaSuccess && nbr > 0x7fffffffull) e = cudaErrorInvalidValue;
    if (e == cudaSuccess) {
      decrypt_poly_kernel<<<dim3((unsigned)nbr, m), 256, N * 8, st>>>(level_in, d_sk, d_sks, ctx->d_tables, N,
                                                                    ps.log_n, m, dm, res);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
      const uint64_t threads = nbr * N;
      lift_pack_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(res, nbr, N, m, bits, lc, dm,
                                                                           (unsigned long long *)out);
      e = cudaGetLastError();
      ctx->launches += 2;
    }
    cudaFreeAsync(res, st);
    // This level's plaintext is the next level's ciphertexts.
    if (d_out) cudaFreeAsync(d_out, st);
    d_out = out;
    level_in = out;
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(plaintext, d_out, aggregated_bytes,
                        out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st);
  cleanup();
  const cudaError_t se = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = se;
  return status_of(e);
}
