/* xpir_oracle.c -- CPU restatement of XPIR's NFLLWE reply path (see xpir_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never part of the product.
 * File:line references are to the XPIR reference sources (v0.2.0-beta).
 */
#include "xpir_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* The 60-bit CRT moduli p_i = 2^61 - i*2^14 + 1, the primitive 2^14-th roots of unity
 * and the inverses of 8192 modulo each p_i.  These must be the reference's exact values
 * (crypto/NFLParams.cpp:30,36,40): every NTT-domain word depends on them. */
static const uint64_t kModuli[XO_MAX_MODULI] = {
    2305843009213317121ULL, 2305843009213120513ULL, 2305843009212694529ULL, 2305843009212399617ULL,
    2305843009211662337ULL, 2305843009211596801ULL, 2305843009211400193ULL, 2305843009210580993ULL,
    2305843009210515457ULL, 2305843009210023937ULL, 2305843009209057281ULL, 2305843009208795137ULL,
    2305843009208713217ULL, 2305843009208123393ULL, 2305843009207468033ULL, 2305843009206976513ULL,
    2305843009206845441ULL};
static const uint64_t kRoots2p14[XO_MAX_MODULI] = {
    1187132827279672845ULL, 753478288701480417ULL,  717492273700781398ULL,  1965831349000139179ULL,
    2188074825493578002ULL, 232964966911499637ULL,  395215708149128273ULL,  241993652537061162ULL,
    370764889455808762ULL,  1598724739621481826ULL, 610870591815427803ULL,  1880981984715338041ULL,
    1389374064030612248ULL, 1508488901479281364ULL, 2111887543055470169ULL, 2020509703903079203ULL,
    1120240637471598814ULL};
static const uint64_t kInv8192[XO_MAX_MODULI] = {
    2305561534236606511ULL, 2305561534236409927ULL, 2305561534235983995ULL, 2305561534235689119ULL,
    2305561534234951929ULL, 2305561534234886401ULL, 2305561534234689817ULL, 2305561534233870717ULL,
    2305561534233805189ULL, 2305561534233313729ULL, 2305561534232347191ULL, 2305561534232085079ULL,
    2305561534232003169ULL, 2305561534231413417ULL, 2305561534230758137ULL, 2305561534230266677ULL,
    2305561534230135621ULL};

uint64_t xo_modulus(uint32_t i) { return i < XO_MAX_MODULI ? kModuli[i] : 0; }

static uint32_t ilog2(uint64_t x) {
  uint32_t r = 0;
  while (x > 1) {
    x >>= 1;
    r++;
  }
  return r;
}

static int valid_shape(uint32_t N, uint32_t m) {
  return m >= 1 && m <= XO_MAX_MODULI && N >= 4 && N <= 8192 && (N & (N - 1)) == 0;
}

/* Full modular product (crypto/NFLlib.hpp:272-275). */
static inline uint64_t mulmod(uint64_t x, uint64_t y, uint64_t p) { return (uint64_t)(((u128)x * y) % p); }

/* Shoup factor floor(y * 2^64 / p), truncated to 64 bits (crypto/NFLlib.hpp:580,
 * pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:764). */
static inline uint64_t shoup(uint64_t y, uint64_t p) { return (uint64_t)(((u128)y << 64) / p); }

/* x*y mod p from the Shoup factor, one final conditional subtraction
 * (crypto/NFLlib.hpp:282-289). */
static inline uint64_t mulmod_shoup(uint64_t x, uint64_t y, uint64_t ys, uint64_t p) {
  uint64_t q = (uint64_t)(((u128)x * ys) >> 64);
  uint64_t r = x * y - q * p;
  return r >= p ? r - p : r;
}

/* Lazy multiply-accumulate: rop += x*y - q*p (mod 2^64), then at most one subtraction of
 * p.  The accumulator is not canonical and its bits depend on the order of the calls
 * (crypto/NFLlib.hpp:303-321). */
static inline uint64_t mac_shoup(uint64_t rop, uint64_t x, uint64_t y, uint64_t ys, uint64_t p) {
  uint64_t q = (uint64_t)(((u128)x * ys) >> 64);
  rop += x * y - q * p;
  return rop >= p ? rop - p : rop;
}

uint64_t xo_tables_words(uint32_t N, uint32_t m) { return (uint64_t)m * (1 + 8 * (uint64_t)N) + N; }

/* Powers of w laid out layer by layer: N/2 powers of w, then N/4 of w^2, ... (the
 * table walk of crypto/NFLlib.hpp:571-586). */
static void layer_powers(uint64_t *tab, uint64_t *tabs, uint64_t w, uint32_t N, uint64_t p) {
  for (uint32_t K = N; K >= 2; K >>= 1) {
    uint64_t wi = 1;
    for (uint32_t i = 0; i < K / 2; i++) {
      *tab++ = wi;
      *tabs++ = shoup(wi, p);
      wi = mulmod(wi, w, p);
    }
    w = mulmod(w, w, p);
  }
  *tab = 0; /* the N-th slot is never written by the reference; keep it defined */
  *tabs = 0;
}

/* crypto/NFLlib.cpp:44-194 (the GMP lifting integers are not needed on this path). */
int xo_tables(uint32_t N, uint32_t m, uint64_t *out) {
  if (!valid_shape(N, m)) return -1;
  const uint32_t logN = ilog2(N);
  uint64_t *o = out;
  for (uint32_t c = 0; c < m; c++) {
    const uint64_t p = kModuli[c];
    uint64_t *phis = o + 1, *phis_s = phis + N, *w = phis_s + N, *w_s = w + N;
    uint64_t *iphis = w_s + N, *iphis_s = iphis + N, *iw = iphis_s + N, *iw_s = iw + N;
    o[0] = p;
    /* phi: the 2^14-th root squared (13 - log2 N) times is a primitive 2N-th root. */
    uint64_t phi = kRoots2p14[c];
    for (int i = 0; i < 13 - (int)logN; i++) phi = mulmod(phi, phi, p);
    uint64_t t = 1;
    for (uint32_t i = 0; i < N; i++) {
      phis[i] = t;
      phis_s[i] = shoup(t, p);
      t = mulmod(t, phi, p);
    }
    /* t = phi^N; phi^N * phi^(N-1) = phi^(2N-1) = phi^-1. */
    const uint64_t invphi = mulmod(t, phis[N - 1], p);
    const uint64_t invN = mulmod(kInv8192[c], 8192 / N, p);
    t = invN;
    for (uint32_t i = 0; i < N; i++) {
      iphis[i] = t;
      iphis_s[i] = shoup(t, p);
      t = mulmod(t, invphi, p);
    }
    layer_powers(w, w_s, mulmod(phi, phi, p), N, p);
    layer_powers(iw, iw_s, mulmod(invphi, invphi, p), N, p);
    o += 1 + 8 * (uint64_t)N;
  }
  /* Bit reversal over log2 N bits; it is an involution, so it is its own inverse. */
  for (uint32_t i = 0; i < N; i++) {
    uint32_t r = 0, ii = i;
    for (uint32_t h = 1; h < N; h <<= 1) {
      r = (r << 1) | (ii & 1);
      ii >>= 1;
    }
    o[i] = r;
  }
  return 0;
}

/* crypto/NFLLWE.cpp:656-668 with noiseUB = 5k/2 (integer) from crypto/NFLLWE.cpp:84. */
uint32_t xo_bits_per_coeff(uint32_t N, uint32_t m, uint32_t k, uint64_t n0) {
  double berr = (double)(uint64_t)(5 * (uint64_t)k / 2);
  double nb_sum = (double)n0;
  double p_size = (double)(60 * m);
  double bits = floor(((p_size - 1) - log2(nb_sum) - log2(berr) - log2((double)N)) / 2.0);
  return bits > 0 ? (uint32_t)bits : 0;
}

/* crypto/NFLlib.cpp:379 (double arithmetic, as the reference). */
uint64_t xo_polys_for_bits(uint64_t total_bits, uint32_t b, uint32_t N) {
  return (uint64_t)ceil((double)total_bits / (double)((uint64_t)b * N));
}

/* nbits (<= 64) bits of the concatenated stream from bit pos; zeros past its end. */
static uint64_t stream_bits(const uint8_t *bufs, uint64_t nbufs, uint64_t stride, uint64_t bpb, uint64_t pos,
                            uint32_t nbits) {
  uint64_t v = 0;
  uint32_t got = 0;
  while (got < nbits) {
    uint64_t bi = pos / bpb;
    if (bi >= nbufs) break;
    uint64_t off = pos - bi * bpb;
    uint64_t avail = bpb - off;
    uint32_t take = nbits - got;
    if (take > avail) take = (uint32_t)avail;
    const uint8_t *p = bufs + bi * stride + (off >> 3);
    uint32_t sh = (uint32_t)(off & 7), nb = (sh + take + 7) / 8;
    u128 w = 0;
    for (uint32_t i = 0; i < nb; i++) w |= (u128)p[i] << (8 * i);
    uint64_t val = (uint64_t)(w >> sh);
    if (take < 64) val &= (1ULL << take) - 1;
    v |= val << got;
    got += take;
    pos += take;
  }
  return v;
}

/* The reference's bit splitter walks the buffers with byte-unaligned 64-bit loads and
 * carries partial sub-chunks across buffer boundaries (crypto/NFLlib.cpp:672-809); its
 * output is that of a plain LSB-first bit stream over the concatenated buffers:
 * coefficient k of poly j is bits [(jN+k)b, (jN+k+1)b), zero past the data.
 * b <= 56: that value, copied to every modulus (crypto/NFLlib.cpp:812-839).
 * b > 56: the value is cut into 56-bit sub-chunks s_t (the last one shorter) and
 * modulus i receives sum_t mulmod(s_t, 2^(56t) mod p_i), each term reduced but the sum
 * not (crypto/NFLlib.cpp:882-916). */
int xo_bitsplit(const uint8_t *bufs, uint64_t nbufs, uint64_t buf_stride, uint64_t bits_per_buffer, uint32_t b,
                uint32_t N, uint32_t m, uint64_t *out) {
  if (!valid_shape(N, m) || b == 0 || b > 56 * 4) return -1;
  const uint64_t total = nbufs * bits_per_buffer;
  const uint64_t P = xo_polys_for_bits(total, b, N);
  const uint32_t nsub = (b + 55) / 56;
  uint64_t mult[XO_MAX_MODULI][4];
  for (uint32_t c = 0; c < m; c++) {
    mult[c][0] = 1;
    for (uint32_t t = 1; t < nsub; t++) mult[c][t] = mulmod(mult[c][t - 1], 1ULL << 56, kModuli[c]);
  }
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < (int64_t)P; j++) {
    for (uint32_t k = 0; k < N; k++) {
      const uint64_t chunk = (uint64_t)j * N + k;
      const uint64_t pos = chunk * b;
      uint64_t *o = out + (uint64_t)j * m * N + k;
      if (nsub == 1) {
        uint64_t v = pos < total ? stream_bits(bufs, nbufs, buf_stride, bits_per_buffer, pos, b) : 0;
        for (uint32_t c = 0; c < m; c++) o[(uint64_t)c * N] = v;
      } else {
        uint64_t sub[4] = {0, 0, 0, 0};
        for (uint32_t t = 0; t < nsub; t++) {
          uint32_t sz = (t + 1 < nsub) ? 56 : b - 56 * (nsub - 1);
          uint64_t sp = pos + 56ULL * t;
          sub[t] = sp < total ? stream_bits(bufs, nbufs, buf_stride, bits_per_buffer, sp, sz) : 0;
        }
        for (uint32_t c = 0; c < m; c++) {
          uint64_t acc = 0;
          for (uint32_t t = 0; t < nsub; t++) acc += mulmod(sub[t], mult[c][t], kModuli[c]);
          o[(uint64_t)c * N] = acc;
        }
      }
    }
  }
  return 0;
}

/* Harvey's lazy decimation-in-frequency NTT as modified by XPIR (crypto/NFLlib.hpp:450-537):
 * log2(N)-2 radix-2 layers with inputs and outputs in [0, 2p), then the last two layers
 * fused per group of four.  Natural order in, bit-reversed order out. */
static void ntt_lazy(uint64_t *x, const uint64_t *w, const uint64_t *ws, uint32_t N, uint64_t p) {
  const uint64_t p2 = 2 * p;
  if (N == 2) {
    uint64_t u0 = x[0], u1 = x[1];
    uint64_t t0 = u0 + u1, t1 = u0 - u1;
    t0 -= (t0 >= p2) ? p2 : 0;
    t1 += ((int64_t)t1 < 0) ? p2 : 0;
    x[0] = t0;
    x[1] = t1;
    return;
  }
  const uint32_t layers = ilog2(N) - 2;
  for (uint32_t l = 0; l < layers; l++) {
    const uint32_t len = N >> l, half = len >> 1;
    for (uint32_t base = 0; base < N; base += len) {
      for (uint32_t i = 0; i < half; i++) {
        uint64_t u0 = x[base + i], u1 = x[base + i + half];
        uint64_t t0 = u0 + u1;
        t0 -= (t0 >= p2) ? p2 : 0;
        uint64_t t1 = u0 - u1 + p2;
        uint64_t q = (uint64_t)(((u128)t1 * ws[i]) >> 64);
        x[base + i] = t0;
        x[base + i + half] = t1 * w[i] - q * p;
      }
    }
    w += half;
    ws += half;
  }
  /* w now points at the 4-point layer: w[1] is the primitive 4th root. */
  for (uint32_t base = 0; base < N; base += 4) {
    uint64_t *y = x + base;
    uint64_t u0 = y[0], u1 = y[1], u2 = y[2], u3 = y[3];
    uint64_t v0 = u0 + u2;
    v0 -= (v0 >= p2) ? p2 : 0;
    uint64_t v2 = u0 - u2;
    v2 += ((int64_t)v2 < 0) ? p2 : 0;
    uint64_t v1 = u1 + u3;
    v1 -= (v1 >= p2) ? p2 : 0;
    uint64_t t = u1 - u3 + p2;
    uint64_t q = (uint64_t)(((u128)t * ws[1]) >> 64);
    uint64_t v3 = t * w[1] - q * p;
    uint64_t z0 = v0 + v1;
    z0 -= (z0 >= p2) ? p2 : 0;
    uint64_t z1 = v0 - v1;
    z1 += ((int64_t)z1 < 0) ? p2 : 0;
    uint64_t z2 = v2 + v3;
    z2 -= (z2 >= p2) ? p2 : 0;
    uint64_t z3 = v2 - v3;
    z3 += ((int64_t)z3 < 0) ? p2 : 0;
    y[0] = z0;
    y[1] = z1;
    y[2] = z2;
    y[3] = z3;
  }
}

int xo_ntt_phi(uint64_t *polys, uint64_t npolys, uint32_t N, uint32_t m) {
  if (!valid_shape(N, m)) return -1;
  uint64_t *tab = (uint64_t *)malloc(xo_tables_words(N, m) * 8);
  if (!tab) return -2;
  xo_tables(N, m, tab);
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < (int64_t)npolys; j++) {
    for (uint32_t c = 0; c < m; c++) {
      const uint64_t *t = tab + (uint64_t)c * (1 + 8 * (uint64_t)N);
      const uint64_t p = t[0], *phis = t + 1, *phis_s = phis + N, *w = phis_s + N, *ws = w + N;
      uint64_t *x = polys + ((uint64_t)j * m + c) * N;
      for (uint32_t i = 0; i < N; i++) x[i] = mulmod_shoup(x[i], phis[i], phis_s[i], p);
      ntt_lazy(x, w, ws, N, p);
    }
  }
  free(tab);
  return 0;
}

/* crypto/NFLlib.hpp:548-566 and 613-626: bit-reverse, forward lazy NTT with the inverse
 * roots, bit-reverse back, then multiply by N^-1 phi^-i (fully reduced). */
int xo_intt_phi(uint64_t *polys, uint64_t npolys, uint32_t N, uint32_t m) {
  if (!valid_shape(N, m)) return -1;
  uint64_t *tab = (uint64_t *)malloc(xo_tables_words(N, m) * 8);
  if (!tab) return -2;
  xo_tables(N, m, tab);
  const uint64_t *rev = tab + (uint64_t)m * (1 + 8 * (uint64_t)N);
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < (int64_t)npolys; j++) {
    uint64_t *y = (uint64_t *)malloc((size_t)N * 8);
    for (uint32_t c = 0; c < m; c++) {
      const uint64_t *t = tab + (uint64_t)c * (1 + 8 * (uint64_t)N);
      const uint64_t p = t[0], *iphis = t + 1 + 4 * (uint64_t)N, *iphis_s = iphis + N;
      const uint64_t *iw = iphis_s + N, *iws = iw + N;
      uint64_t *x = polys + ((uint64_t)j * m + c) * N;
      for (uint32_t i = 0; i < N; i++) y[rev[i]] = x[i];
      ntt_lazy(y, iw, iws, N, p);
      for (uint32_t i = 0; i < N; i++) x[rev[i]] = y[i];
      for (uint32_t i = 0; i < N; i++) x[i] = mulmod_shoup(x[i], iphis[i], iphis_s[i], p);
    }
    free(y);
  }
  free(tab);
  return 0;
}

/* The reference fills one reused buffer per aggregated element s (importDataNFL calls
 * readAggregatedStream for s = 0, 1, ... on the same calloc'd buffer,
 * PIRReplyGeneratorNFL_internal.cpp:88,104-106).  For a group cut short by the end of the
 * database (r < alpha real elements) the zero fill starts at slot r-1, not r, and stops
 * at slot alpha-2 (DBHandler.cpp:21-24): slot r-1 (the last real element) reads as
 * zeros and slot alpha-1 keeps what the previous group left there (element s*alpha-1,
 * or zeros for s = 0). */
void xo_aggregate(const uint8_t *elements, uint64_t nb_elements, uint64_t element_bytes, uint64_t element_stride,
                  uint32_t alpha, uint64_t s, uint8_t *out) {
  const uint64_t first = s * alpha;
  const uint64_t end = (first + alpha - 1 < nb_elements - 1) ? first + alpha - 1 : nb_elements - 1;
  const uint64_t padding = (first + alpha >= nb_elements) ? first + alpha - nb_elements : 0;
  for (uint64_t i = first; i <= end; i++)
    memcpy(out + (i % alpha) * element_bytes, elements + i * element_stride, element_bytes);
  if (padding != 0) {
    /* r = alpha - padding real elements sit in slots 0..r-1; the reference zeroes slots
     * r-1 .. alpha-2 and never writes slot alpha-1 in this call, which therefore keeps
     * the previous (full) group's last element, or the calloc zeros when s = 0. */
    const uint64_t stale = alpha - 1;
    if (s > 0)
      memcpy(out + stale * element_bytes, elements + (first - 1) * element_stride, element_bytes);
    else
      memset(out + stale * element_bytes, 0, element_bytes);
    memset(out + (end % alpha) * element_bytes, 0, element_bytes * padding);
  }
}

int xo_import(const uint8_t *elements, uint64_t nb_elements, uint64_t element_bytes, uint64_t element_stride,
              uint32_t alpha, uint32_t b, uint32_t N, uint32_t m, uint64_t *out) {
  if (!valid_shape(N, m) || alpha == 0 || nb_elements == 0) return -1;
  if (b == 0 || b > 56 * 4) return -1;
  const uint64_t groups = (nb_elements + alpha - 1) / alpha;
  const uint64_t bits = 8 * (uint64_t)alpha * element_bytes;
  const uint64_t P = xo_polys_for_bits(bits, b, N);
  int failed = 0;
  /* Aggregated elements are independent (xo_aggregate reproduces the reused buffer's
   * state from the element indexes alone), so they are split in parallel. */
#pragma omp parallel reduction(| : failed)
  {
    uint8_t *agg = (uint8_t *)malloc(alpha * element_bytes + 16);
    if (!agg) failed = 1;
#pragma omp for schedule(dynamic, 16)
    for (int64_t s = 0; s < (int64_t)groups; s++) {
      if (!agg) continue;
      xo_aggregate(elements, nb_elements, element_bytes, element_stride, alpha, (uint64_t)s, agg);
      if (xo_bitsplit(agg, 1, bits / 8 + 16, bits, b, N, m, out + (uint64_t)s * P * m * N)) failed = 1;
    }
    free(agg);
  }
  if (failed) return -2;
  return xo_ntt_phi(out, groups * P, N, m);
}

void xo_query_primes(const uint64_t *y, uint64_t n, uint32_t N, uint32_t m, uint64_t *out) {
  for (uint64_t i = 0; i < n; i++)
    for (uint32_t h = 0; h < 2; h++)
      for (uint32_t c = 0; c < m; c++)
        for (uint32_t k = 0; k < N; k++) {
          uint64_t idx = ((i * 2 + h) * m + c) * N + k;
          out[idx] = shoup(y[idx], kModuli[c]);
        }
}

int xo_reply_level(const uint64_t *db, uint64_t n_real, uint64_t P, uint64_t n_groups, uint64_t n_i,
                   const uint64_t *query, uint32_t N, uint32_t m, uint64_t *out) {
  if (!valid_shape(N, m)) return -1;
  const uint64_t mN = (uint64_t)m * N, ct = 2 * mN;
  const uint32_t KB = 64; /* coefficients per work item */
  const uint32_t nkb = N / KB;
  /* Chains are independent per (group, poly, half, modulus, coefficient); each one runs
   * over the slots of its group strictly in order.  The query Shoup factors
   * (pushQuery, PIRReplyGeneratorNFL_internal.cpp:756-767) are recomputed per use. */
#pragma omp parallel for collapse(4) schedule(dynamic, 1)
  for (int64_t j = 0; j < (int64_t)n_groups; j++) {
    for (int64_t cp = 0; cp < (int64_t)P; cp++) {
      for (int64_t c = 0; c < (int64_t)m; c++) {
        for (int64_t kb = 0; kb < (int64_t)nkb; kb++) {
          const uint64_t p = kModuli[c];
          const uint64_t k0 = (uint64_t)kb * KB;
          uint64_t *ra = out + ((uint64_t)j * P + cp) * ct + c * N + k0;
          uint64_t *rb = ra + mN;
          memset(ra, 0, KB * 8);
          memset(rb, 0, KB * 8);
          /* A group made only of padding slots adds x = 0 terms (t = 0) to a zero start:
           * its reply stays exactly zero. */
          if ((uint64_t)j * n_i >= n_real) continue;
          for (uint64_t q = 0; q < n_i; q++) {
            const uint64_t e = (uint64_t)j * n_i + q;
            const uint64_t *ya = query + q * ct + c * N + k0, *yb = ya + mN;
            /* a slot past the real elements is an all-zero element
             * (PIRReplyGeneratorNFL_internal.cpp:146-154) */
            const uint64_t *x = e < n_real ? db + (e * P + cp) * mN + c * N + k0 : NULL;
            for (uint32_t k = 0; k < KB; k++) {
              const uint64_t xk = x ? x[k] : 0;
              ra[k] = mac_shoup(ra[k], xk, ya[k], shoup(ya[k], p), p);
              rb[k] = mac_shoup(rb[k], xk, yb[k], shoup(yb[k], p), p);
            }
          }
        }
      }
    }
  }
  return 0;
}

int xo_reimport(const uint64_t *replies, uint64_t n_elts, uint64_t P, uint32_t b, uint32_t N, uint32_t m,
                uint64_t *out) {
  if (!valid_shape(N, m)) return -1;
  const uint64_t ct_words = 2ULL * m * N, ct_bits = 64 * ct_words;
  const uint64_t P2 = xo_polys_for_bits(P * ct_bits, b, N);
  int failed = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(| : failed)
  for (int64_t e = 0; e < (int64_t)n_elts; e++) {
    if (xo_bitsplit((const uint8_t *)(replies + (uint64_t)e * P * ct_words), P, ct_words * 8, ct_bits, b, N, m,
                    out + (uint64_t)e * P2 * m * N))
      failed = 1;
  }
  if (failed) return -1;
  return xo_ntt_phi(out, n_elts * P2, N, m);
}

uint64_t xo_reply(const uint64_t *db, uint64_t n_real, uint64_t P, uint32_t d, const uint32_t *n,
                  const uint64_t *query, uint32_t b, uint32_t N, uint32_t m, uint64_t *out) {
  if (!valid_shape(N, m) || d == 0) return 0;
  const uint64_t mN = (uint64_t)m * N, ct_words = 2 * mN;
  const uint64_t *in = db;
  uint64_t *owned = NULL;
  uint64_t in_real = n_real, in_P = P;
  for (uint32_t lvl = 0; lvl < d; lvl++) {
    uint64_t groups = 1;
    for (uint32_t j = lvl + 1; j < d; j++) groups *= n[j];
    uint64_t *rep = (uint64_t *)malloc(groups * in_P * ct_words * 8);
    if (!rep) {
      free(owned);
      return 0;
    }
    xo_reply_level(in, in_real, in_P, groups, n[lvl], query, N, m, rep);
    query += (uint64_t)n[lvl] * ct_words;
    free(owned);
    owned = NULL;
    if (lvl + 1 == d) {
      memcpy(out, rep, in_P * ct_words * 8);
      free(rep);
      return in_P;
    }
    const uint64_t P2 = xo_polys_for_bits(in_P * 64 * ct_words, b, N);
    owned = (uint64_t *)malloc(groups * P2 * mN * 8);
    if (!owned) {
      free(rep);
      return 0;
    }
    xo_reimport(rep, groups, in_P, b, N, m, owned);
    free(rep);
    in = owned;
    in_real = groups;
    in_P = P2;
  }
  return 0;
}

/* computeReplySizeInChunks: ceil over doubles per level, as the reference. */
uint64_t xo_reply_count(uint64_t element_bytes, uint32_t alpha, uint32_t d, uint32_t b, uint32_t N, uint32_t m) {
  const double abs_bits = (double)((uint64_t)b * N);
  unsigned int out = (unsigned int)ceil((double)element_bytes * 8 * alpha / abs_bits);
  const uint64_t ct_bytes = 2ULL * 64 * m * N / 8;
  const uint64_t abs_bytes = (uint64_t)b * N / 8;
  for (uint32_t i = 1; i < d; i++) out = (unsigned int)ceil(out * (double)ct_bytes / (double)abs_bytes);
  return out;
}

/* ---- client-side decryption and extraction ---------------------------------------- */

static uint64_t powmod(uint64_t a, uint64_t e, uint64_t p) {
  uint64_t r = 1;
  a %= p;
  while (e) {
    if (e & 1) r = mulmod(r, a, p);
    a = mulmod(a, a, p);
    e >>= 1;
  }
  return r;
}

/* Multi-word helpers (little-endian 64-bit limbs, XO_LIMBS of them). */
#define XO_LIMBS 6
static uint64_t limbs_mod(const uint64_t *x, uint64_t p) {
  u128 r = 0;
  for (int i = XO_LIMBS - 1; i >= 0; i--) r = ((r << 64) | x[i]) % p;
  return (uint64_t)r;
}
static void limbs_muladd(uint64_t *x, const uint64_t *M, uint64_t v) { /* x += M*v */
  u128 carry = 0;
  for (int i = 0; i < XO_LIMBS; i++) {
    u128 t = (u128)M[i] * v + x[i] + carry;
    x[i] = (uint64_t)t;
    carry = t >> 64;
  }
}
static void limbs_mul_small(uint64_t *M, uint64_t v) { /* M *= v */
  u128 carry = 0;
  for (int i = 0; i < XO_LIMBS; i++) {
    u128 t = (u128)M[i] * v + carry;
    M[i] = (uint64_t)t;
    carry = t >> 64;
  }
}
static int limbs_cmp(const uint64_t *a, const uint64_t *b) {
  for (int i = XO_LIMBS - 1; i >= 0; i--)
    if (a[i] != b[i]) return a[i] > b[i] ? 1 : -1;
  return 0;
}

/* NFLLWE::dec + NFLLWE::decrypt for one ciphertext (crypto/NFLLWE.cpp:375-475, 515-551):
 * per modulus m_c = submod(b_c, mulandaddShoup(0, a_c, s_c), p_c) (NFLlib.hpp:255-267,
 * 303-321), inverse NTT and N^-1 phi^-i (NFLlib.hpp:613-626), then per coefficient the CRT
 * lift x in [0, P) (NFLlib.cpp:504-532; computed here by mixed radix, which gives the same
 * unique x), centred: x - P when 2x > P, and its low b bits, serialised LSB-first
 * (NFLlib.cpp:412-495).  out receives b*N/8 bytes. */
int xo_decrypt(const uint64_t *ct, const uint64_t *sk, uint32_t b, uint32_t N, uint32_t m, uint8_t *out) {
  if (!valid_shape(N, m) || b == 0 || b >= 128 || (uint64_t)b >= 61ull * m) return -1;
  uint64_t *tab = (uint64_t *)malloc(xo_tables_words(N, m) * 8);
  uint64_t *mm = (uint64_t *)malloc((size_t)m * N * 8);
  if (!tab || !mm) {
    free(tab);
    free(mm);
    return -2;
  }
  xo_tables(N, m, tab);
  for (uint32_t c = 0; c < m; c++) {
    const uint64_t p = tab[(uint64_t)c * (1 + 8 * (uint64_t)N)];
    const uint64_t *a = ct + (uint64_t)c * N, *bb = ct + ((uint64_t)m + c) * N, *s = sk + (uint64_t)c * N;
    for (uint32_t i = 0; i < N; i++) {
      const uint64_t temp = mac_shoup(0, a[i], s[i], shoup(s[i], p), p);
      const uint64_t y = (temp < p) ? p - temp : p - temp % p;
      uint64_t z = bb[i] + y;
      z -= (z >= p) ? p : 0;
      mm[(uint64_t)c * N + i] = z;
    }
  }
  xo_intt_phi(mm, 1, N, m);
  /* CRT constants: P, and for mixed radix the prefix products and their inverses. */
  uint64_t P[XO_LIMBS] = {1}, Mi[XO_MAX_MODULI][XO_LIMBS], inv[XO_MAX_MODULI];
  for (uint32_t c = 0; c < m; c++) {
    const uint64_t p = xo_modulus(c);
    memcpy(Mi[c], P, sizeof(P));
    inv[c] = c ? powmod(limbs_mod(P, p), p - 2, p) : 1;
    limbs_mul_small(P, p);
  }
  memset(out, 0, (size_t)b * N / 8);
  for (uint32_t i = 0; i < N; i++) {
    uint64_t x[XO_LIMBS] = {0};
    for (uint32_t c = 0; c < m; c++) {
      const uint64_t p = xo_modulus(c);
      const uint64_t r = mm[(uint64_t)c * N + i] % p;
      const uint64_t have = limbs_mod(x, p);
      const uint64_t v = mulmod((r + p - have) % p, inv[c], p);
      limbs_muladd(x, Mi[c], v);
    }
    uint64_t x2[XO_LIMBS];
    uint64_t carry = 0;
    for (int k = 0; k < XO_LIMBS; k++) {
      x2[k] = (x[k] << 1) | carry;
      carry = x[k] >> 63;
    }
    uint64_t lo = x[0], hi = x[1];
    if (limbs_cmp(x2, P) > 0) { /* x - P mod 2^128 */
      const u128 d = (((u128)x[1] << 64) | x[0]) - (((u128)P[1] << 64) | P[0]);
      lo = (uint64_t)d;
      hi = (uint64_t)(d >> 64);
    }
    /* low b bits at bit offset i*b */
    const uint64_t pos = (uint64_t)i * b;
    for (uint32_t k = 0; k < b; k++) {
      const uint64_t bit = k < 64 ? (lo >> k) & 1 : (hi >> (k - 64)) & 1;
      if (bit) out[(pos + k) >> 3] |= (uint8_t)(1u << ((pos + k) & 7));
    }
  }
  free(tab);
  free(mm);
  return 0;
}

/* Ciphertexts decrypted at recursion level lvl (1 = the innermost) for an aggregated
 * element of agg_bytes: PIRReplyExtraction_internal::extractReply's float arithmetic
 * (pir/replyExtraction/PIRReplyExtraction_internal.cpp:50-58). */
uint64_t xo_extract_count(uint64_t agg_bytes, uint32_t lvl, uint32_t b, uint32_t N, uint32_t m) {
  const float abs_bytes = (float)((uint64_t)b * N / 8), ct_bytes = (float)(16ull * m * N);
  uint64_t nbr = (uint64_t)ceilf((float)agg_bytes / abs_bytes);
  for (uint32_t i = 1; i < lvl; i++) nbr = (uint64_t)ceilf((float)nbr * ct_bytes / abs_bytes);
  return nbr;
}

/* PIRReplyExtraction_internal::extractReply (…_internal.cpp:41-106): from level d down
 * to 1, decrypt that level's ciphertexts (the replies at d; below, the previous level's
 * plaintext bytes read as ciphertexts); the level-1 plaintexts concatenated give the
 * aggregated element, of which agg_bytes are written to out. */
int xo_extract(const uint64_t *replies, uint64_t nb_replies, const uint64_t *sk, uint32_t d, uint32_t b, uint32_t N,
               uint32_t m, uint64_t agg_bytes, uint8_t *out) {
  const uint64_t abs_bytes = (uint64_t)b * N / 8, ct_words = 2ull * m * N;
  if (d == 0 || abs_bytes == 0) return -1;
  if (nb_replies < xo_extract_count(agg_bytes, d, b, N, m)) return -1;
  uint8_t *in = NULL; /* plaintext of the level above, read as ciphertexts */
  for (uint32_t lvl = d; lvl >= 1; lvl--) {
    const uint64_t nbr = xo_extract_count(agg_bytes, lvl, b, N, m);
    uint8_t *plain = (uint8_t *)calloc(nbr * abs_bytes + 8, 1);
    if (!plain) {
      free(in);
      return -2;
    }
    for (uint64_t j = 0; j < nbr; j++) {
      const uint64_t *c = lvl == d ? replies + j * ct_words : (const uint64_t *)(in + j * ct_words * 8);
      if (xo_decrypt(c, sk, b, N, m, plain + j * abs_bytes) != 0) {
        free(plain);
        free(in);
        return -1;
      }
    }
    free(in);
    in = plain;
  }
  memcpy(out, in, agg_bytes);
  free(in);
  return 0;
}

/* ---- client-side query generation --------------------------------------------------- */

/* Salsa20/20 keystream (the published algorithm; the reference calls NaCl's
 * crypto_stream_salsa20 through fastrandombytes, crypto/prng/fastrandombytes.cpp:34-55):
 * 64-byte blocks of the state (constants, 256-bit key, 64-bit nonce, 64-bit block counter
 * from 0) after 20 rounds plus the input, little-endian. */
#define XO_ROTL(v, c) (((v) << (c)) | ((v) >> (32 - (c))))
static void salsa20_block(const uint32_t in[16], uint8_t out[64]) {
  uint32_t x[16];
  memcpy(x, in, sizeof(x));
  for (int r = 0; r < 10; r++) {
    x[4] ^= XO_ROTL(x[0] + x[12], 7);   x[8] ^= XO_ROTL(x[4] + x[0], 9);
    x[12] ^= XO_ROTL(x[8] + x[4], 13);  x[0] ^= XO_ROTL(x[12] + x[8], 18);
    x[9] ^= XO_ROTL(x[5] + x[1], 7);    x[13] ^= XO_ROTL(x[9] + x[5], 9);
    x[1] ^= XO_ROTL(x[13] + x[9], 13);  x[5] ^= XO_ROTL(x[1] + x[13], 18);
    x[14] ^= XO_ROTL(x[10] + x[6], 7);  x[2] ^= XO_ROTL(x[14] + x[10], 9);
    x[6] ^= XO_ROTL(x[2] + x[14], 13);  x[10] ^= XO_ROTL(x[6] + x[2], 18);
    x[3] ^= XO_ROTL(x[15] + x[11], 7);  x[7] ^= XO_ROTL(x[3] + x[15], 9);
    x[11] ^= XO_ROTL(x[7] + x[3], 13);  x[15] ^= XO_ROTL(x[11] + x[7], 18);
    x[1] ^= XO_ROTL(x[0] + x[3], 7);    x[2] ^= XO_ROTL(x[1] + x[0], 9);
    x[3] ^= XO_ROTL(x[2] + x[1], 13);   x[0] ^= XO_ROTL(x[3] + x[2], 18);
    x[6] ^= XO_ROTL(x[5] + x[4], 7);    x[7] ^= XO_ROTL(x[6] + x[5], 9);
    x[4] ^= XO_ROTL(x[7] + x[6], 13);   x[5] ^= XO_ROTL(x[4] + x[7], 18);
    x[11] ^= XO_ROTL(x[10] + x[9], 7);  x[8] ^= XO_ROTL(x[11] + x[10], 9);
    x[9] ^= XO_ROTL(x[8] + x[11], 13);  x[10] ^= XO_ROTL(x[9] + x[8], 18);
    x[12] ^= XO_ROTL(x[15] + x[14], 7); x[13] ^= XO_ROTL(x[12] + x[15], 9);
    x[14] ^= XO_ROTL(x[13] + x[12], 13); x[15] ^= XO_ROTL(x[14] + x[13], 18);
  }
  for (int i = 0; i < 16; i++) {
    const uint32_t v = x[i] + in[i];
    out[4 * i] = (uint8_t)v;
    out[4 * i + 1] = (uint8_t)(v >> 8);
    out[4 * i + 2] = (uint8_t)(v >> 16);
    out[4 * i + 3] = (uint8_t)(v >> 24);
  }
}

static uint32_t le32(const uint8_t *b) { return (uint32_t)b[0] | (uint32_t)b[1] << 8 | (uint32_t)b[2] << 16 | (uint32_t)b[3] << 24; }

void xo_salsa20_stream(uint8_t *out, uint64_t len, uint64_t nonce, const uint8_t key[32]) {
  uint32_t in[16];
  in[0] = 0x61707865u; in[5] = 0x3320646eu; in[10] = 0x79622d32u; in[15] = 0x6b206574u;  /* "expand 32-byte k" */
  for (int i = 0; i < 4; i++) {
    in[1 + i] = le32(key + 4 * i);
    in[11 + i] = le32(key + 16 + 4 * i);
  }
  in[6] = (uint32_t)nonce;
  in[7] = (uint32_t)(nonce >> 32);
  uint8_t block[64];
  for (uint64_t ctr = 0, off = 0; off < len; ctr++, off += 64) {
    in[8] = (uint32_t)ctr;
    in[9] = (uint32_t)(ctr >> 32);
    salsa20_block(in, block);
    memcpy(out + off, block, len - off < 64 ? (size_t)(len - off) : 64);
  }
}

/* mask = 2^ceil(log2(bound)) - 1 with the reference's double arithmetic (NFLlib.cpp:305,339) */
static uint64_t bound_mask(uint64_t bound) { return (1ULL << (unsigned int)ceil(log2((double)bound))) - 1; }

/* NFLlib::setBoundedRandomPoly in uniform mode (crypto/NFLlib.cpp:325-353): one
 * fastrandombytes call of m*N words (nonce `nonce`), masked and reduced per modulus. */
static void uniform_poly(const uint8_t key[32], uint64_t nonce, uint32_t N, uint32_t m, uint64_t *out) {
  xo_salsa20_stream((uint8_t *)out, (uint64_t)m * N * 8, nonce, key);
  for (uint32_t c = 0; c < m; c++) {
    const uint64_t p = xo_modulus(c), mask = bound_mask(p);
    for (uint32_t i = 0; i < N; i++) {
      uint64_t r = out[(uint64_t)c * N + i] & mask;
      if (r >= p) r -= p;
      out[(uint64_t)c * N + i] = r;
    }
  }
}

/* NFLLWE's secret key (crypto/NFLLWE.cpp:108-116): a uniform poly from the PRNG call with
 * the given nonce (the first call, nonce 0, for a fresh crypto object). */
int xo_keygen(const uint8_t key[32], uint64_t nonce, uint32_t N, uint32_t m, uint64_t *sk) {
  if (!valid_shape(N, m)) return -1;
  uniform_poly(key, nonce, N, m, sk);
  return 0;
}

/* NFLLWE::encrypt(ui) -> enc (crypto/NFLLWE.cpp:276-372, 481-498) with the PRNG calls at
 * nonces `nonce` (the noise, N words, NFLlib.cpp:290-321) and nonce+1 (the uniform a):
 * b = NTT_phi(e*2^b mod p + m) + a*s, with e in [0, 2*(5k/2)-1) and m = ui on the
 * constant coefficient of every modulus. */
int xo_encrypt(const uint8_t key[32], uint64_t nonce, const uint64_t *sk, uint32_t ui, uint32_t b, uint32_t k,
               uint32_t N, uint32_t m, uint64_t *ct) {
  if (!valid_shape(N, m)) return -1;
  uint64_t *a = ct, *bb = ct + (uint64_t)m * N;
  const uint64_t ub = 2 * (5 * (uint64_t)k / 2) - 1, nmask = bound_mask(ub);
  uint64_t *noise = (uint64_t *)malloc((size_t)N * 8);
  if (!noise) return -2;
  xo_salsa20_stream((uint8_t *)noise, (uint64_t)N * 8, nonce, key);
  for (uint32_t i = 0; i < N; i++) {
    noise[i] &= nmask;
    if (noise[i] >= ub) noise[i] -= ub;
  }
  for (uint32_t c = 0; c < m; c++) {
    const uint64_t p = xo_modulus(c);
    const uint64_t amp = (uint64_t)(((u128)1 << b) % p);  /* 2^b mod p (b < 128) */
    const uint64_t amps = shoup(amp, p);
    for (uint32_t i = 0; i < N; i++) {
      uint64_t v = mulmod_shoup(noise[i], amp, amps, p);
      uint64_t z = v + (i == 0 ? ui : 0);
      z -= (z >= p) ? p : 0;   /* addmod */
      if (z > p) z -= p;
      bb[(uint64_t)c * N + i] = z;
    }
  }
  free(noise);
  xo_ntt_phi(bb, 1, N, m);
  uniform_poly(key, nonce + 1, N, m, a);
  for (uint32_t c = 0; c < m; c++) {
    const uint64_t p = xo_modulus(c);
    /* with SHOUP defined (crypto/NFLLWE.hpp:21) both halves leave fully reduced
     * (crypto/NFLLWE.cpp:355-358) */
    for (uint64_t i = (uint64_t)c * N; i < (uint64_t)(c + 1) * N; i++) {
      bb[i] = mac_shoup(bb[i], a[i], sk[i], shoup(sk[i], p), p) % p;
      a[i] %= p;
    }
  }
  return 0;
}

/* PIRQueryGenerator_internal::generateQuery (pir/queryGen/PIRQueryGenerator_internal.cpp:37-70):
 * for level j, n[j] encryptions of [i == coord_j] where coord is the chosen element in
 * mixed radix n[0], n[1], ...; ciphertext t uses nonces first_nonce + 2t and + 2t + 1. */
int xo_query(const uint8_t key[32], uint64_t first_nonce, const uint64_t *sk, uint32_t d, const uint32_t *n,
             uint64_t chosen, uint32_t b, uint32_t k, uint32_t N, uint32_t m, uint64_t *out) {
  uint64_t t = 0, x = chosen;
  const uint64_t ct_words = 2ull * m * N;
  for (uint32_t j = 0; j < d; j++) {
    const uint64_t coord = x % n[j];
    x /= n[j];
    for (uint64_t i = 0; i < n[j]; i++, t++)
      if (xo_encrypt(key, first_nonce + 2 * t, sk, i == coord ? 1u : 0u, b, k, N, m, out + t * ct_words) != 0)
        return -1;
  }
  return 0;
}
