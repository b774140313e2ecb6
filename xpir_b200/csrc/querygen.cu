// Client-side query generation on the GPU: the ciphertexts PIRQueryGenerator builds
// (pir/queryGen/PIRQueryGenerator_internal.cpp:37-70), with NFLLWE::encrypt's arithmetic
// (crypto/NFLLWE.cpp:276-372, 481-498) and the randomness of the reference's PRNG: every
// fastrandombytes call (crypto/prng/fastrandombytes.cpp:34-55) is a Salsa20/20 keystream
// from block 0 under the client's 32-byte key, with a 64-bit nonce that counts the calls.
// Each ciphertext makes two calls, the noise (N words) then the uniform a (m*N words), so
// ciphertext t of a query uses nonces first + 2t and first + 2t + 1; Salsa20 being a
// counter-mode stream, every 64-byte block is computed independently on the device.
//
// encrypt_kernel: one CTA per ciphertext.  The noise is drawn once (its words are below
// the noise bound, so they are kept as 32-bit words in shared memory) and serves every
// modulus; then per modulus:
//   e   = noise word amplified by 2^b mod p (Shoup), plus the plaintext bit on the
//         constant coefficient;
//   b   = NTT(phi-twist(e + m)) with the import's lazy NTT (outputs in [0, 2p));
//   a   = uniform word & mask, minus p when above it (so a < p);
//   b  += a*s (lazy Shoup MAC: [0, 3p)), then both halves fully reduced (SHOUP is defined
//         in the reference, crypto/NFLLWE.hpp:21, crypto/NFLLWE.cpp:355-358): a already
//         is, b by two conditional subtractions (2p, then p), which is b mod p for b < 4p.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

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

struct QueryGenArgs {
  uint32_t key[8];            // Salsa20 key words (little-endian)
  uint64_t first_nonce;
  uint64_t one_slot[XPIR_B200_MAX_LEVELS];  // global index of the ciphertext encrypting 1, per level
  uint32_t d;
  uint64_t noise_bound, noise_mask;
  uint64_t amp[kMaxModuli], amp_shoup[kMaxModuli], uniform_mask[kMaxModuli];
};

__device__ __forceinline__ uint32_t rotl32(uint32_t v, int c) { return (v << c) | (v >> (32 - c)); }

// One 64-byte Salsa20/20 block as 16 little-endian words.
__device__ __forceinline__ void salsa20_block(const uint32_t key[8], uint64_t nonce, uint64_t counter,
                                              uint32_t out[16]) {
  uint32_t in[16];
  in[0] = 0x61707865u;  // "expand 32-byte k"
  in[5] = 0x3320646eu;
  in[10] = 0x79622d32u;
  in[15] = 0x6b206574u;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    in[1 + i] = key[i];
    in[11 + i] = key[4 + i];
  }
  in[6] = (uint32_t)nonce;
  in[7] = (uint32_t)(nonce >> 32);
  in[8] = (uint32_t)counter;
  in[9] = (uint32_t)(counter >> 32);
  uint32_t x[16];
#pragma unroll
  for (int i = 0; i < 16; i++) x[i] = in[i];
#pragma unroll 2
  for (int r = 0; r < 10; r++) {
    x[4] ^= rotl32(x[0] + x[12], 7);   x[8] ^= rotl32(x[4] + x[0], 9);
    x[12] ^= rotl32(x[8] + x[4], 13);  x[0] ^= rotl32(x[12] + x[8], 18);
    x[9] ^= rotl32(x[5] + x[1], 7);    x[13] ^= rotl32(x[9] + x[5], 9);
    x[1] ^= rotl32(x[13] + x[9], 13);  x[5] ^= rotl32(x[1] + x[13], 18);
    x[14] ^= rotl32(x[10] + x[6], 7);  x[2] ^= rotl32(x[14] + x[10], 9);
    x[6] ^= rotl32(x[2] + x[14], 13);  x[10] ^= rotl32(x[6] + x[2], 18);
    x[3] ^= rotl32(x[15] + x[11], 7);  x[7] ^= rotl32(x[3] + x[15], 9);
    x[11] ^= rotl32(x[7] + x[3], 13);  x[15] ^= rotl32(x[11] + x[7], 18);
    x[1] ^= rotl32(x[0] + x[3], 7);    x[2] ^= rotl32(x[1] + x[0], 9);
    x[3] ^= rotl32(x[2] + x[1], 13);   x[0] ^= rotl32(x[3] + x[2], 18);
    x[6] ^= rotl32(x[5] + x[4], 7);    x[7] ^= rotl32(x[6] + x[5], 9);
    x[4] ^= rotl32(x[7] + x[6], 13);   x[5] ^= rotl32(x[4] + x[7], 18);
    x[11] ^= rotl32(x[10] + x[9], 7);  x[8] ^= rotl32(x[11] + x[10], 9);
    x[9] ^= rotl32(x[8] + x[11], 13);  x[10] ^= rotl32(x[9] + x[8], 18);
    x[12] ^= rotl32(x[15] + x[14], 7); x[13] ^= rotl32(x[12] + x[15], 9);
    x[14] ^= rotl32(x[13] + x[12], 13); x[15] ^= rotl32(x[14] + x[13], 18);
  }
#pragma unroll
  for (int i = 0; i < 16; i++) out[i] = x[i] + in[i];
}

__global__ void __launch_bounds__(256, 4) encrypt_kernel(const QueryGenArgs g, const uint64_t *__restrict__ sk,
                                                      const uint64_t *__restrict__ sks,
                                                      const uint64_t *__restrict__ tables, uint32_t N, uint32_t log_n,
                                                      uint32_t m, const DevModuli dm, uint64_t *__restrict__ out) {
  extern __shared__ uint64_t poly[];                     // N words, swizzled (the NTT's buffer)
  uint32_t *noise = reinterpret_cast<uint32_t *>(poly + N);  // N words, [k][blk] (conflict-free)
  const uint32_t nb = N / 8;                             // Salsa20 blocks of 8 words per poly
  const uint64_t t = blockIdx.x;
  uint64_t ui = 0;
  for (uint32_t l = 0; l < g.d; l++) ui |= (g.one_slot[l] == t) ? 1 : 0;
  const uint64_t nonce_e = g.first_nonce + 2 * t, nonce_a = nonce_e + 1;
  // noise e (the same words for every modulus): word & mask, minus the bound when above it
  for (uint32_t blk = threadIdx.x; blk < nb; blk += blockDim.x) {
    uint32_t w[16];
    salsa20_block(g.key, nonce_e, blk, w);
#pragma unroll
    for (int k = 0; k < 8; k++) {
      uint64_t r = ((uint64_t)w[2 * k] | (uint64_t)w[2 * k + 1] << 32) & g.noise_mask;
      if (r >= g.noise_bound) r -= g.noise_bound;
      noise[k * nb + blk] = (uint32_t)r;  // read back by this thread only
    }
  }
  for (uint32_t c = 0; c < m; c++) {
    const uint64_t p = dm.p[c], p2 = p << 1;
    const uint64_t *tab = tables + (uint64_t)c * kTableSlots * N;
    const uint64_t *phi = tab + kPhi * N, *phis = tab + kPhiShoup * N;
    // amplified, plus the plaintext, twisted
    for (uint32_t blk = threadIdx.x; blk < nb; blk += blockDim.x) {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const uint32_t i = blk * 8 + k;
        uint64_t z = shoup_mul(noise[k * nb + blk], g.amp[c], g.amp_shoup[c], p) + (i == 0 ? ui : 0);
        z -= (z >= p) ? p : 0;
        if (z > p) z -= p;
        poly[swz(i)] = shoup_mul(z, phi[i], phis[i], p);
      }
    }
    __syncthreads();
    ntt_lazy_rb<3>(poly, tab + kOmega * N, tab + kOmegaShoup * N, N, log_n, p,
                   [&](uint32_t k) { return poly[swz(k)]; });
    // uniform a: words [c*N, (c+1)*N) of the second call's stream
    uint64_t *a_out = out + (t * 2 * m + c) * N, *b_out = out + (t * 2 * m + m + c) * N;
    const uint64_t *s = sk + (uint64_t)c * N, *ss = sks + (uint64_t)c * N;
    for (uint32_t blk = threadIdx.x; blk < nb; blk += blockDim.x) {
      uint32_t w[16];
      salsa20_block(g.key, nonce_a, (uint64_t)c * nb + blk, w);
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const uint32_t i = blk * 8 + k;
        uint64_t a = ((uint64_t)w[2 * k] | (uint64_t)w[2 * k + 1] << 32) & g.uniform_mask[c];
        if (a >= p) a -= p;
        uint64_t b = shoup_mac(poly[swz(i)], a, s[i], ss[i], p);
        b -= (b >= p2) ? p2 : 0;
        b -= (b >= p) ? p : 0;
        a_out[i] = a;
        b_out[i] = b;
      }
    }
    __syncthreads();  // the next modulus rewrites poly
  }
}

// The secret key's Shoup factors floor(s*2^64/p) (s < p), on the device.
__global__ void __launch_bounds__(256) key_shoup_kernel(const uint64_t *__restrict__ sk, uint64_t *__restrict__ sks,
                                                        uint32_t N, const DevModuli dm) {
  const uint32_t c = blockIdx.y;
  const uint64_t p = dm.p[c];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    sks[(uint64_t)c * N + i] = shoup_factor8_np(sk[(uint64_t)c * N + i], p, 0 - p, (uint32_t)dm.shoup_delta[c]);
}

// NFLLWE's secret key (crypto/NFLLWE.cpp:108-116): the uniform poly of one PRNG call.
__global__ void __launch_bounds__(256) keygen_kernel(const QueryGenArgs g, uint64_t nonce, uint32_t N,
                                                     const DevModuli dm, uint64_t *__restrict__ sk) {
  const uint32_t c = blockIdx.y;
  const uint64_t p = dm.p[c];
  for (uint32_t blk = blockIdx.x * blockDim.x + threadIdx.x; blk < N / 8; blk += gridDim.x * blockDim.x) {
    uint32_t w[16];
    salsa20_block(g.key, nonce, (uint64_t)c * (N / 8) + blk, w);
#pragma unroll
    for (int k = 0; k < 8; k++) {
      uint64_t a = ((uint64_t)w[2 * k] | (uint64_t)w[2 * k + 1] << 32) & g.uniform_mask[c];
      if (a >= p) a -= p;
      sk[(uint64_t)c * N + blk * 8 + k] = a;
    }
  }
}

int status_of(cudaError_t e) {
  if (e == cudaSuccess) return XPIR_B200_OK;
  (void)cudaGetLastError();
  if (e == cudaErrorMemoryAllocation) return XPIR_B200_ERR_NOMEM;
  return XPIR_B200_ERR_CUDA;
}

// 2^ceil(log2(bound)) - 1 with the reference's double arithmetic (crypto/NFLlib.cpp:305,339).
uint64_t bound_mask(uint64_t bound) { return (1ULL << (unsigned int)std::ceil(std::log2((double)bound))) - 1; }

}  // namespace

cudaError_t launch_key_shoup(const uint64_t *sk, uint64_t *sks, uint32_t N, uint32_t m, const DevModuli &dm,
                             cudaStream_t stream) {
  key_shoup_kernel<<<dim3((N + 255) / 256, m), 256, 0, stream>>>(sk, sks, N, dm);
  return cudaGetLastError();
}

}  // namespace xpir

using namespace xpir;

extern "C" int xpir_b200_generate_query(xpir_b200_ctx *ctx, const uint8_t *prng_key, uint64_t first_nonce,
                                        const uint64_t *secret_key, uint32_t d, const uint32_t *n,
                                        uint64_t chosen_element, uint32_t bits_per_coeff, uint32_t security_bits,
                                        void *query, uint64_t capacity_bytes, int out_on_device) {
  if (!ctx || !prng_key || !secret_key || !n || !query || d == 0 || d > XPIR_B200_MAX_LEVELS || bits_per_coeff == 0 ||
      bits_per_coeff >= 128 || security_bits == 0)
    return XPIR_B200_ERR_ARG;
  const ParamSet &ps = ctx->ps;
  const uint32_t N = ps.N, m = ps.m;
  const uint64_t mN = (uint64_t)m * N, ct_bytes = 2 * mN * 8;
  uint64_t nq = 0;
  for (uint32_t j = 0; j < d; j++) {
    if (n[j] == 0) return XPIR_B200_ERR_ARG;
    nq += n[j];
  }
  if (capacity_bytes < nq * ct_bytes || nq > 0x7fffffffull) return XPIR_B200_ERR_ARG;
  QueryGenArgs g;
  memset(&g, 0, sizeof(g));
  for (int i = 0; i < 8; i++)
    g.key[i] = (uint32_t)prng_key[4 * i] | (uint32_t)prng_key[4 * i + 1] << 8 | (uint32_t)prng_key[4 * i + 2] << 16 |
               (uint32_t)prng_key[4 * i + 3] << 24;
  g.first_nonce = first_nonce;
  g.d = d;
  // computeCoordinates (PIRQueryGenerator_internal.cpp:76-85): mixed radix n[0], n[1], ...
  uint64_t x = chosen_element, base = 0;
  for (uint32_t j = 0; j < d; j++) {
    g.one_slot[j] = base + x % n[j];
    x /= n[j];
    base += n[j];
  }
  g.noise_bound = 2 * (5 * (uint64_t)security_bits / 2) - 1;  // 2*Berr - 1, Berr = 5k/2 (NFLLWE.cpp:83)
  g.noise_mask = bound_mask(g.noise_bound);
  if (g.noise_mask >= (1ULL << 32)) return XPIR_B200_ERR_ARG;  // the kernel keeps noise words in 32 bits
  for (uint32_t c = 0; c < m; c++) {
    const uint64_t p = ps.mod[c].p;
    g.amp[c] = (uint64_t)((((unsigned __int128)1) << bits_per_coeff) % p);  // 2^b mod p (NFLLWE.cpp:590-604)
    g.amp_shoup[c] = (uint64_t)(((unsigned __int128)g.amp[c] << 64) / p);
    g.uniform_mask[c] = bound_mask(p);
  }
  const DevModuli dm = make_dev_moduli(ps);

  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return status_of(e);
  cudaStream_t st = ctx->stream;
  uint64_t *d_sk = nullptr, *d_sks = nullptr, *d_out = nullptr;
  e = cudaMallocFromPoolAsync((void **)&d_sk, mN * 8, ctx->pool, st);
  if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void **)&d_sks, mN * 8, ctx->pool, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_sk, secret_key, mN * 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    e = launch_key_shoup(d_sk, d_sks, N, m, dm, st);
    ctx->launches++;
  }
  uint64_t *target = (uint64_t *)query;
  if (e == cudaSuccess && !out_on_device) {
    e = cudaMallocFromPoolAsync((void **)&d_out, nq * ct_bytes, ctx->pool, st);
    target = d_out;
  }
  const int smem = (int)(N * 8 + N * 4);  // the NTT's poly and the 32-bit noise words
  if (e == cudaSuccess) e = allow_max_dynamic_smem((const void *)encrypt_kernel);
  if (e == cudaSuccess) {
    encrypt_kernel<<<(unsigned)nq, 256, smem, st>>>(g, d_sk, d_sks, ctx->d_tables, N, ps.log_n, m, dm, target);
    e = cudaGetLastError();
    ctx->launches++;
  }
  if (e == cudaSuccess && !out_on_device) e = cudaMemcpyAsync(query, d_out, nq * ct_bytes, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d_sk, st);
  cudaFreeAsync(d_sks, st);
  if (d_out) cudaFreeAsync(d_out, st);
  const cudaError_t se = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = se;
  return status_of(e);
}

extern "C" int xpir_b200_generate_secret_key(xpir_b200_ctx *ctx, const uint8_t *prng_key, uint64_t nonce,
                                             uint64_t *secret_key) {
  if (!ctx || !prng_key || !secret_key) return XPIR_B200_ERR_ARG;
  const ParamSet &ps = ctx->ps;
  const uint64_t mN = (uint64_t)ps.m * ps.N;
  QueryGenArgs g;
  memset(&g, 0, sizeof(g));
  for (int i = 0; i < 8; i++)
    g.key[i] = (uint32_t)prng_key[4 * i] | (uint32_t)prng_key[4 * i + 1] << 8 | (uint32_t)prng_key[4 * i + 2] << 16 |
               (uint32_t)prng_key[4 * i + 3] << 24;
  for (uint32_t c = 0; c < ps.m; c++) g.uniform_mask[c] = bound_mask(ps.mod[c].p);
  const DevModuli dm = make_dev_moduli(ps);
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return status_of(e);
  cudaStream_t st = ctx->stream;
  uint64_t *d_sk = nullptr;
  e = cudaMallocFromPoolAsync((void **)&d_sk, mN * 8, ctx->pool, st);
  if (e == cudaSuccess) {
    keygen_kernel<<<dim3((ps.N / 8 + 255) / 256, ps.m), 256, 0, st>>>(g, nonce, ps.N, dm, d_sk);
    e = cudaGetLastError();
    ctx->launches++;
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(secret_key, d_sk, mN * 8, cudaMemcpyDeviceToHost, st);
  if (d_sk) cudaFreeAsync(d_sk, st);
  const cudaError_t se = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = se;
  return status_of(e);
}
