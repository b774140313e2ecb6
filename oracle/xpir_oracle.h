/* xpir_oracle: CPU restatement of XPIR's NFLLWE reply path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared against; it
 * is never linked into, called by, or used as a fallback for the product library.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm load it.
 *
 * Every function restates one piece of the reference (file:line given per function).
 * Its outputs are pinned against the reference's own code, compiled unchanged by
 * oracle/Makefile (target `ref`), and against the committed fixtures in tests/golden/.
 *
 * Layouts (all little-endian u64):
 *   polynomial  [m][N]                 modulus-major, then coefficient
 *   ciphertext  [2][m][N]              a then b
 *   imported DB [elements][P][m][N]
 *   query       [n_level][2][m][N]     one ciphertext per slot, level by level
 */
#ifndef XPIR_ORACLE_H
#define XPIR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XO_MAX_MODULI 17

/* The i-th 60-bit CRT modulus (crypto/NFLParams.cpp:28-30). */
uint64_t xo_modulus(uint32_t i);

/* NTT tables for (N, m), laid out per modulus as
 * [p][phi^i N][phi' N][omega tab N][omega' N][N^-1 phi^-i N][shoup N][omega^-1 tab N][shoup N]
 * followed once by the inverse bit-reversal indexes [N].  (crypto/NFLlib.cpp:44-194) */
int xo_tables(uint32_t N, uint32_t m, uint64_t *out);
uint64_t xo_tables_words(uint32_t N, uint32_t m);

/* Bits absorbed per coefficient for security k and first dimension n0
 * (crypto/NFLLWE.cpp:656-668, noise bound 5k/2 from crypto/NFLLWE.cpp:84). */
uint32_t xo_bits_per_coeff(uint32_t N, uint32_t m, uint32_t k, uint64_t n0);

/* Polynomials needed to absorb total_bits at b bits per coefficient
 * (crypto/NFLlib.cpp:379). */
uint64_t xo_polys_for_bits(uint64_t total_bits, uint32_t b, uint32_t N);

/* Bit splitter + CRT: nbufs buffers of bits_per_buffer bits (buffer i starts at
 * bufs + i*buf_stride), read as one LSB-first bit stream, cut into b-bit coefficients.
 * out receives P*m*N words, P = xo_polys_for_bits(nbufs*bits_per_buffer, b, N).
 * (crypto/NFLlib.cpp:672-916) */
int xo_bitsplit(const uint8_t *bufs, uint64_t nbufs, uint64_t buf_stride, uint64_t bits_per_buffer,
                uint32_t b, uint32_t N, uint32_t m, uint64_t *out);

/* phi-twist + forward NTT, in place, on npolys polynomials of m*N words
 * (crypto/NFLlib.hpp:597-608 -> 450-537). */
int xo_ntt_phi(uint64_t *polys, uint64_t npolys, uint32_t N, uint32_t m);

/* Inverse NTT + inverse phi-twist, in place (crypto/NFLlib.hpp:613-626 -> 548-566). */
int xo_intt_phi(uint64_t *polys, uint64_t npolys, uint32_t N, uint32_t m);

/* Aggregated element s of a database of nb_elements elements (element i at
 * elements + i*element_stride, element_bytes used), alpha elements per group, as the
 * reference's DBHandler::readAggregatedStream leaves its reused buffer when called for
 * s = 0, 1, ... in order (pir/dbhandlers/DBHandler.cpp:3-26,
 * pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:88,104-106).  out: alpha*element_bytes. */
void xo_aggregate(const uint8_t *elements, uint64_t nb_elements, uint64_t element_bytes,
                  uint64_t element_stride, uint32_t alpha, uint64_t s, uint8_t *out);

/* Database import: aggregation, bit split, CRT and NTT of every aggregated element.
 * out: ceil(nb_elements/alpha) * P * m * N words, P = xo_polys_for_bits(8*alpha*element_bytes, b, N).
 * (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:79-158) */
int xo_import(const uint8_t *elements, uint64_t nb_elements, uint64_t element_bytes, uint64_t element_stride,
              uint32_t alpha, uint32_t b, uint32_t N, uint32_t m, uint64_t *out);

/* Shoup precomputation of query words: floor(y * 2^64 / p) mod 2^64
 * (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:756-767).  y: n ciphertexts. */
void xo_query_primes(const uint64_t *y, uint64_t n, uint32_t N, uint32_t m, uint64_t *out);

/* One recursion level of the reply: for group j < n_groups and poly cp < P, the
 * ciphertext accumulated in order over the n_i slots of the group, slot q taking DB
 * element j*n_i + q (an all-zero element when that index is >= n_real).
 * out: n_groups * P * 2*m*N words.
 * (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:511-595, crypto/NFLLWE.cpp:176-205,
 *  crypto/NFLlib.hpp:303-321) */
int xo_reply_level(const uint64_t *db, uint64_t n_real, uint64_t P, uint64_t n_groups, uint64_t n_i,
                   const uint64_t *query, uint32_t N, uint32_t m, uint64_t *out);

/* Re-import of level replies as the next level's database: element e's P ciphertexts
 * are one bit stream of P buffers of 2*64*m*N bits.  out: n_elts * P2 * m * N words,
 * P2 = xo_polys_for_bits(P*128*m*N, b, N).
 * (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:599-626) */
int xo_reimport(const uint64_t *replies, uint64_t n_elts, uint64_t P, uint32_t b, uint32_t N, uint32_t m,
                uint64_t *out);

/* Full reply for d levels over an imported level-0 database of n_real elements with P
 * polys each; query holds sum(n) ciphertexts.  Writes the final replies (P_last
 * ciphertexts) to out and returns P_last, or 0 on error.
 * (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:340-445) */
uint64_t xo_reply(const uint64_t *db, uint64_t n_real, uint64_t P, uint32_t d, const uint32_t *n,
                  const uint64_t *query, uint32_t b, uint32_t N, uint32_t m, uint64_t *out);

/* Number of final reply ciphertexts (computeReplySizeInChunks,
 * pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:667-679). */
uint64_t xo_reply_count(uint64_t element_bytes, uint32_t alpha, uint32_t d, uint32_t b, uint32_t N, uint32_t m);

/* Client-side decryption of one ciphertext with the secret key sk ([m][N], NTT domain,
 * as NFLLWE::secretKey holds it): b*N/8 plaintext bytes (crypto/NFLLWE.cpp:375-475,
 * 515-551). */
int xo_decrypt(const uint64_t *ct, const uint64_t *sk, uint32_t b, uint32_t N, uint32_t m, uint8_t *out);

/* Ciphertexts decrypted at recursion level lvl for agg_bytes of aggregated element
 * (PIRReplyExtraction_internal.cpp:50-58). */
uint64_t xo_extract_count(uint64_t agg_bytes, uint32_t lvl, uint32_t b, uint32_t N, uint32_t m);

/* Reply extraction for d levels (PIRReplyExtraction_internal.cpp:41-106): agg_bytes of
 * the aggregated element into out.  0 on success. */
int xo_extract(const uint64_t *replies, uint64_t nb_replies, const uint64_t *sk, uint32_t d, uint32_t b, uint32_t N,
               uint32_t m, uint64_t agg_bytes, uint8_t *out);

/* Client-side query generation.  Salsa20/20 keystream for one fastrandombytes call
 * (crypto/prng/fastrandombytes.cpp:34-55): len bytes, 64-bit nonce, 32-byte key. */
void xo_salsa20_stream(uint8_t *out, uint64_t len, uint64_t nonce, const uint8_t key[32]);
/* NFLLWE's secret key from the PRNG call with the given nonce (crypto/NFLLWE.cpp:108-116). */
int xo_keygen(const uint8_t key[32], uint64_t nonce, uint32_t N, uint32_t m, uint64_t *sk);
/* NFLLWE::encrypt(ui) with the noise at nonce and the uniform a at nonce+1
 * (crypto/NFLLWE.cpp:276-372, 481-498). */
int xo_encrypt(const uint8_t key[32], uint64_t nonce, const uint64_t *sk, uint32_t ui, uint32_t b, uint32_t k,
               uint32_t N, uint32_t m, uint64_t *ct);
/* The sum(n) query ciphertexts for the chosen element (PIRQueryGenerator_internal.cpp:37-70). */
int xo_query(const uint8_t key[32], uint64_t first_nonce, const uint64_t *sk, uint32_t d, const uint32_t *n,
             uint64_t chosen, uint32_t b, uint32_t k, uint32_t N, uint32_t m, uint64_t *out);

#ifdef __cplusplus
}
#endif

#endif
