// Database import on the GPU: aggregation, bit split, CRT, phi-twist and the lazy
// decimation-in-frequency NTT, fused in one kernel per (aggregated element, poly, modulus).
//
// Reference path (crypto/NFLlib.cpp:375-401, 672-916; crypto/NFLlib.hpp:450-537, 597-608;
// pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:79-158).  The same kernel performs
// the re-import of level replies between recursion levels (…NFL_internal.cpp:599-626):
// the P reply ciphertexts of an element are one contiguous little-endian bit stream.
//
// HBM layout of the output: [element][poly][modulus][coefficient] u64, values in [0, 2p).
#include <cuda_runtime.h>
#include <algorithm>
#include <stdint.h>

#include "kernels.h"
#include "modarith.cuh"
#include "ntt.cuh"

namespace xpir {

DevModuli make_dev_moduli(const ParamSet &ps) {
  DevModuli d{};
  for (uint32_t c = 0; c < ps.m; c++) {
    d.p[c] = ps.mod[c].p;
    d.shoup_k[c] = ps.mod[c].shoup_k;
    d.shoup_delta[c] = ps.mod[c].shoup_delta;
    for (int t = 0; t < 4; t++) {
      d.crt[c][t] = ps.mod[c].crt[t];
      d.crt_shoup[c][t] = ps.mod[c].crt_shoup[t];
    }
  }
  return d;
}

namespace {

// Threads per import CTA: N/16, two 8-coefficient groups of the register-blocked NTT
// per thread and pass (on B200 this beat one group per thread, 16-coefficient groups,
// and the transform fed straight from the bit extraction, all bit-identical).
constexpr uint32_t kImportMaxThreads = kMaxPolyDegree / 16;
inline uint32_t import_threads(uint32_t N) { return N / 16; }

struct ImportShape {
  uint32_t N, log_n, m, b, nsub;
  uint64_t P;
  uint64_t per_row, active;  // element s of CTA u = blockIdx.x / P: (u / active) * per_row + u % active
  uint64_t total_bytes;  // bytes of one aggregated element (alpha * element_bytes)
  uint32_t stage_words;  // u64 words of staged input per poly
};

// Byte i of aggregated element s, following the reference's reused import buffer: a
// short last group (r < alpha real elements) reads its last real slot r-1 and slots up
// to alpha-2 as zeros, and slot alpha-1 as the previous group's last element (zeros for
// the first group).  See oracle xo_aggregate and pir/dbhandlers/DBHandler.cpp:3-26.
__device__ __forceinline__ uint8_t agg_byte(const AggSource &src, uint64_t s, uint64_t i, uint64_t real) {
  const uint64_t slot = i / src.element_bytes, off = i - slot * src.element_bytes;
  const uint64_t first = s * src.alpha;
  uint64_t elem;
  if (real == src.alpha) {
    elem = first + slot;
  } else if (slot + 1 < real) {
    elem = first + slot;
  } else if (slot + 1 == src.alpha) {
    if (s == 0) return 0;
    elem = first - 1;
  } else {
    return 0;
  }
  return src.base[elem * src.element_stride + off];
}


// nbits (<= 56) bits starting at bit `pos` of the staged little-endian words.
__device__ __forceinline__ uint64_t staged_bits(const uint64_t *st, uint64_t pos, uint32_t nbits) {
  const uint64_t w = pos >> 6;
  const uint32_t sh = (uint32_t)(pos & 63);
  uint64_t v = st[w] >> sh;
  if (sh) v |= st[w + 1] << (64 - sh);
  return v & ((1ull << nbits) - 1);
}

// grid: x = aggregated element * P + poly, y = modulus; import_threads(N) threads.
// Dynamic smem: stage words, then N words.
__global__ void __launch_bounds__(kImportMaxThreads) import_kernel(const AggSource src, const ImportShape sh,
                                                                   const DevModuli dm,
                                                                   const uint64_t *__restrict__ tables,
                                                                   uint64_t *__restrict__ out) {
  extern __shared__ __align__(16) uint64_t smem[];
  uint64_t *stage = smem;
  uint64_t *poly = smem + sh.stage_words;
  const uint64_t u = blockIdx.x / sh.P, j = blockIdx.x - u * sh.P;
  const uint64_t row = u / sh.active, s = row * sh.per_row + (u - row * sh.active);
  const uint32_t c = blockIdx.y;
  const uint32_t N = sh.N;
  const uint64_t p = dm.p[c];

  // Stage the bytes of this poly's bit range, from an 8-byte aligned start.
  const uint64_t bit0 = j * (uint64_t)N * sh.b;
  const uint64_t byte0 = (bit0 >> 3) & ~7ull;
  const uint64_t first = s * src.alpha;
  const uint64_t real = (first + src.alpha <= src.nb_elements) ? src.alpha : src.nb_elements - first;
  const bool flat = (real == src.alpha) && (src.alpha == 1 || src.element_stride == src.element_bytes);
  const uint8_t *flat_base = src.base + first * src.element_stride;
  const bool aligned = flat && ((((uintptr_t)flat_base) & 7) == 0);
  for (uint32_t w = threadIdx.x; w < sh.stage_words; w += blockDim.x) {
    const uint64_t bpos = byte0 + 8ull * w;
    uint64_t v = 0;
    if (bpos + 8 <= sh.total_bytes && aligned) {
      v = *reinterpret_cast<const uint64_t *>(flat_base + bpos);
    } else {
      for (uint32_t q = 0; q < 8; q++) {
        const uint64_t i = bpos + q;
        if (i < sh.total_bytes) {
          const uint8_t byte = flat ? flat_base[i] : agg_byte(src, s, i, real);
          v |= (uint64_t)byte << (8 * q);
        }
      }
    }
    stage[w] = v;
  }
  __syncthreads();

  // Coefficient k, twisted by phi^k: b <= 56 one chunk per coefficient; b > 56 sub-chunks
  // of 56 bits combined per modulus as sum_t mulmod(s_t, 2^(56t)) without a final
  // reduction.
  const uint64_t *tab = tables + (uint64_t)c * kTableSlots * N;
  const uint64_t *phi = tab + kPhi * N, *phi_s = tab + kPhiShoup * N;
  const uint64_t rel0 = bit0 - 8 * byte0;
  for (uint32_t k = threadIdx.x; k < N; k += blockDim.x) {
    const uint64_t pos = rel0 + (uint64_t)k * sh.b;
    uint64_t x;
    if (sh.nsub == 1) {
      x = staged_bits(stage, pos, sh.b);
    } else {
      x = 0;
      for (uint32_t t = 0; t < sh.nsub; t++) {
        const uint32_t sz = (t + 1 < sh.nsub) ? 56 : sh.b - 56 * (sh.nsub - 1);
        const uint64_t sub = staged_bits(stage, pos + 56ull * t, sz);
        x += shoup_mul(sub, dm.crt[c][t], dm.crt_shoup[c][t], p);
      }
    }
    poly[swz(k)] = shoup_mul(x, __ldg(phi + k), __ldg(phi_s + k), p);
  }
  __syncthreads();
  ntt_lazy_rb<3>(poly, tab + kOmega * N, tab + kOmegaShoup * N, N, sh.log_n, p,
                 [&](uint32_t k) { return poly[swz(k)]; });

  // Coalesced 16-byte stores; swz(2t+1) == swz(2t) ^ 1.
  ulonglong2 *o = reinterpret_cast<ulonglong2 *>(out + ((s * sh.P + j) * sh.m + c) * (uint64_t)N);
  for (uint32_t t = threadIdx.x; t < N / 2; t += blockDim.x) {
    const uint32_t at = swz(2 * t);
    o[t] = make_ulonglong2(poly[at], poly[at ^ 1]);
  }
}

// The import of an all-zero bit stream, broadcast: every coefficient chunk is 0, so the
// twisted coefficients are 0 and the lazy NTT leaves one fixed poly per modulus (values
// 0 and p).  Each CTA computes it for modulus blockIdx.y in shared memory, then writes it
// to its share of the `count` known-zero polys t (element row * per_row + active +
// (t / P) % (per_row - active) of row t / (P * (per_row - active)), poly t % P).
__global__ void __launch_bounds__(kImportMaxThreads) import_zero_fill_kernel(const ImportShape sh,
                                                                             const DevModuli dm,
                                                                             const uint64_t *__restrict__ tables,
                                                                             uint64_t *__restrict__ out,
                                                                             uint64_t count) {
  extern __shared__ __align__(16) uint64_t smem[];
  const uint32_t c = blockIdx.y, N = sh.N;
  const uint64_t p = dm.p[c];
  const uint64_t *tab = tables + (uint64_t)c * kTableSlots * N;
  const uint64_t *phi = tab + kPhi * N, *phi_s = tab + kPhiShoup * N;
  auto coefficient = [&](uint32_t k) -> uint64_t { return shoup_mul(0, __ldg(phi + k), __ldg(phi_s + k), p); };
  ntt_lazy_rb<3>(smem, tab + kOmega * N, tab + kOmegaShoup * N, N, sh.log_n, p, coefficient);
  const uint64_t zeros = sh.per_row - sh.active;
  for (uint64_t t = blockIdx.x; t < count; t += gridDim.x) {
    const uint64_t u = t / sh.P, j = t - u * sh.P;
    const uint64_t row = u / zeros, s = row * sh.per_row + sh.active + (u - row * zeros);
    ulonglong2 *o = reinterpret_cast<ulonglong2 *>(out + ((s * sh.P + j) * sh.m + c) * (uint64_t)N);
    for (uint32_t i = threadIdx.x; i < N / 2; i += blockDim.x) {
      const uint32_t at = swz(2 * i);
      o[i] = make_ulonglong2(smem[at], smem[at ^ 1]);
    }
  }
}

}  // namespace

cudaError_t launch_import(const AggSource &src, uint64_t groups, uint64_t P, const ParamSet &ps,
                          const DevModuli &dm, const uint64_t *tables, uint64_t *out, cudaStream_t stream,
                          const ImportRows *rows, uint32_t *launches) {
  if (groups == 0 || P == 0) return cudaSuccess;
  const ImportRows r = rows ? *rows : ImportRows{1, groups, groups};
  if (r.rows == 0 || r.per_row == 0 || r.rows * r.per_row != groups || r.active > r.per_row)
    return cudaErrorInvalidValue;
  ImportShape sh;
  sh.N = ps.N;
  sh.log_n = ps.log_n;
  sh.m = ps.m;
  sh.b = ps.b;
  sh.nsub = (ps.b + 55) / 56;
  sh.P = P;
  sh.per_row = r.per_row;
  sh.active = r.active;
  sh.total_bytes = (uint64_t)src.alpha * src.element_bytes;
  // bits of one poly plus the in-word offset, rounded up, plus one spare word for the
  // two-word reads of staged_bits
  sh.stage_words = (uint32_t)((64 + (uint64_t)ps.N * ps.b + 63) / 64 + 2);
  const size_t smem = (size_t)(sh.stage_words + ps.N) * sizeof(uint64_t);
  const unsigned threads = import_threads(ps.N);
  const uint64_t computed = r.rows * r.active, zero_polys = r.rows * (r.per_row - r.active) * P;
  if (computed * P > 0x7fffffffull) return cudaErrorInvalidValue;
  if (computed > 0) {
    cudaError_t e = allow_max_dynamic_smem((const void *)import_kernel);
    if (e != cudaSuccess) return e;
    dim3 grid((unsigned)(computed * P), ps.m);
    import_kernel<<<grid, threads, smem, stream>>>(src, sh, dm, tables, out);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (launches) (*launches)++;
  }
  if (zero_polys > 0) {
    const size_t zsmem = (size_t)ps.N * sizeof(uint64_t);
    cudaError_t e = allow_max_dynamic_smem((const void *)import_zero_fill_kernel);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    // About four CTAs per SM over all moduli: each computes the constant poly once.
    const uint64_t per_mod = std::max<uint64_t>(1, 4ull * (uint64_t)sms / ps.m);
    dim3 grid((unsigned)std::min<uint64_t>(zero_polys, per_mod), ps.m);
    import_zero_fill_kernel<<<grid, threads, zsmem, stream>>>(sh, dm, tables, out, zero_polys);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (launches) (*launches)++;
  }
  return cudaSuccess;
}

// Loads both import kernels on the current device (lazy module loading would otherwise do
// it, and reserve their device memory, at their first launch).
cudaError_t preload_import_kernels() {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, import_kernel);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, import_zero_fill_kernel);
  return e;
}

}  // namespace xpir
