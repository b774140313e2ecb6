/* xpir_b200.h -- C ABI of the B200 (sm_100a) reply engine for XPIR's NFLLWE path.
 *
 * The drop-in boundary: XPIR's PIRReplyGeneratorNFL_internal (the engine behind libpir's
 * PIRReplyGenerator, GenericPIRReplyGenerator and PIRReplyGeneratorFactory("LWE")) is
 * replaced by calls to these functions.  Plain pointers and sizes only; every function
 * returns an XPIR_B200_* status (0 = success) and never aborts the process.
 *
 * Data formats are XPIR's, unchanged (little-endian u64 words):
 *   query ciphertext  [a: m polys x N][b: m polys x N]   getCiphertextBitsize()/8 bytes
 *                     (crypto/NFLLWEPublicParameters.cpp:82-86,148-151)
 *   reply ciphertext  same layout, lazily reduced words, bit-identical to XPIR's
 *   a query           the sum(n[i]) ciphertexts in push order (level 0 slots first),
 *                     back to back, as PIRReplyGeneratorNFL_internal::pushQuery receives
 *                     them (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:722-781)
 *   database          nb_elements elements of element_bytes bytes, element i at
 *                     elements + i*element_stride (the bytes DBHandler::readStream yields)
 */
#ifndef XPIR_B200_H
#define XPIR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define XPIR_B200_API __attribute__((visibility("default")))
#else
#define XPIR_B200_API
#endif

#define XPIR_B200_OK 0
#define XPIR_B200_ERR_ARG (-1)     /* invalid argument or unsupported shape */
#define XPIR_B200_ERR_NOMEM (-2)   /* device or pinned-host allocation failed */
#define XPIR_B200_ERR_CUDA (-3)    /* CUDA runtime error (see xpir_b200_last_cuda_error) */
#define XPIR_B200_ERR_NODEV (-4)   /* no usable CUDA device */
#define XPIR_B200_ERR_STATE (-5)   /* call out of order (e.g. incomplete query) */
#define XPIR_B200_ERR_TIMEOUT (-6) /* a kernel's bounded wait expired; outputs are invalid */
#define XPIR_B200_MAX_LEVELS 10    /* MAX_REC_LVL, pir/PIRParameters.hpp:22 */

typedef struct xpir_b200_ctx xpir_b200_ctx; /* one (N, moduli) parameter set on one GPU */
typedef struct xpir_b200_db xpir_b200_db;   /* an imported database resident in HBM */

/* ---- library ------------------------------------------------------------------ */
XPIR_B200_API const char *xpir_b200_version(void);
XPIR_B200_API const char *xpir_b200_strerror(int status);
/* Name of the last CUDA error seen by the calling thread's calls (diagnostics); for a
 * served query, xpir_b200_server_wait reports the query's CUDA error to its caller. */
XPIR_B200_API const char *xpir_b200_last_cuda_error(void);
XPIR_B200_API int xpir_b200_device_count(int *count);

/* ---- sizing (host only; no GPU needed) ---------------------------------------- */
/* Bits absorbed per coefficient for a query whose first dimension is n0:
 * replaces NFLLWE::setandgetAbsBitPerCiphertext (crypto/NFLLWE.cpp:656-668). */
XPIR_B200_API int32_t xpir_b200_bits_per_coeff(uint32_t poly_degree, uint32_t nb_moduli, uint32_t security_bits, uint64_t n0);
/* Polynomials per (aggregated) element: NFLlib::deserializeDataNFL's polyNumber
 * (crypto/NFLlib.cpp:379). */
XPIR_B200_API uint64_t xpir_b200_polys_per_element(uint64_t element_bytes, uint32_t alpha, uint32_t bits_per_coeff,
                                     uint32_t poly_degree);
/* Number of reply ciphertexts: PIRReplyGeneratorNFL_internal::computeReplySizeInChunks
 * (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:667-679). */
XPIR_B200_API uint64_t xpir_b200_reply_count(uint64_t element_bytes, uint32_t alpha, uint32_t d, uint32_t bits_per_coeff,
                               uint32_t poly_degree, uint32_t nb_moduli);
/* The i-th 60-bit CRT modulus, 2^61 - i*2^14 + 1 (NFLlib::getmoduli, crypto/NFLParams.cpp:30);
 * 0 when i is out of range. */
XPIR_B200_API uint64_t xpir_b200_modulus(uint32_t i);
/* Bytes of one query/reply ciphertext: NFLLWEPublicParameters::getCiphertextBitsize()/8
 * (crypto/NFLLWEPublicParameters.cpp:148-151). */
XPIR_B200_API uint64_t xpir_b200_ciphertext_bytes(uint32_t poly_degree, uint32_t nb_moduli);

/* ---- context -------------------------------------------------------------------- */
/* Parameter set "LWE:k:N:60*nb_moduli" on `device`: builds and uploads the NTT tables,
 * the role of NFLlib::setNewParameters/configureNTT (crypto/NFLlib.cpp:44-228).  The
 * context owns one CUDA stream; all its work is ordered on it. */
XPIR_B200_API int xpir_b200_ctx_create(xpir_b200_ctx **ctx, int device, uint32_t poly_degree, uint32_t nb_moduli);
/* Destroys the context and every database imported through it (their handles become
 * invalid and must not be passed to xpir_b200_db_free afterwards).  XPIR_B200_ERR_STATE,
 * and nothing destroyed, while a server has a lane on the context: destroy it first. */
XPIR_B200_API int xpir_b200_ctx_destroy(xpir_b200_ctx *ctx);
/* The context's cudaStream_t, as a void pointer (for event timing by the caller). */
XPIR_B200_API int xpir_b200_ctx_stream(xpir_b200_ctx *ctx, void **stream);
/* Blocks until all work queued on the context has finished. */
XPIR_B200_API int xpir_b200_ctx_synchronize(xpir_b200_ctx *ctx);
/* Number of engine kernels launched on this context so far. */
XPIR_B200_API int xpir_b200_ctx_launch_count(xpir_b200_ctx *ctx, uint64_t *count);
/* Test support for the reply kernel's bounded waits; no counterpart in the reference.
 * Every wait in the reply kernel gives up after a fixed number of polls (about 2.6 s),
 * records the failure and lets the kernel return, so that a stalled pipeline ends in
 * XPIR_B200_ERR_TIMEOUT instead of a hang.  For the following xpir_b200_reply calls on
 * this context: spin_limit > 0 shortens the limit of the consumers' waits and of the copy
 * producer's ring (the producer's final wait for its own copies in flight keeps the full
 * limit), and withhold_tile >= 0 makes every reply CTA's copy producer stop before that
 * tile's copies, so that the waits for it run out and the call returns
 * XPIR_B200_ERR_TIMEOUT with nothing left in flight.  (0, -1) restores normal operation. */
XPIR_B200_API int xpir_b200_ctx_set_wait_test(xpir_b200_ctx *ctx, uint32_t spin_limit, int32_t withhold_tile);
/* Measurement support; no counterpart in the reference.  on != 0: the following
 * xpir_b200_reply calls on this context record a CUDA event pair on the context's stream
 * around each level's reply launch and each re-import between levels, and add the
 * elapsed times up after the call's synchronisation; the sums restart at zero.  on == 0
 * stops recording (the sums are kept).  Other entry points are not timed. */
XPIR_B200_API int xpir_b200_ctx_set_kernel_timing(xpir_b200_ctx *ctx, int on);
/* The sums of xpir_b200_ctx_set_kernel_timing: reply_ms[l] / reply_launches[l] for
 * recursion level l (XPIR_B200_MAX_LEVELS entries each, level 0 first), and the
 * re-imports' import_ms / import_launches.  Any pointer may be NULL. */
XPIR_B200_API int xpir_b200_ctx_kernel_time(xpir_b200_ctx *ctx, double *reply_ms, uint64_t *reply_launches,
                                            double *import_ms, uint64_t *import_launches);

/* ---- database import -------------------------------------------------------------- */
/* Imports a database for queries whose aggregation is `alpha` and whose first dimension
 * gives `bits_per_coeff`: aggregation as DBHandler::readAggregatedStream, bit split,
 * CRT and NTT as NFLlib::deserializeDataNFL, for every aggregated element.  Replaces
 * PIRReplyGeneratorNFL_internal::importDataNFL (…NFL_internal.cpp:79-158) behind
 * libpir's PIRReplyGenerator::importData (pir/libpir.cpp:90-103).  `elements` is host
 * memory when src_on_device == 0, device memory otherwise.  The zero padding of the
 * index grid (…NFL_internal.cpp:146-154) is not materialised. */
XPIR_B200_API int xpir_b200_db_import(xpir_b200_ctx *ctx, const void *elements, uint64_t nb_elements, uint64_t element_bytes,
                        uint64_t element_stride, uint32_t alpha, uint32_t bits_per_coeff, int src_on_device,
                        xpir_b200_db **db);
/* Frees the device copy: the role of imported_database::~imported_database
 * (pir/libpir.cpp:5-11). */
XPIR_B200_API int xpir_b200_db_free(xpir_b200_db *db);
/* Aggregated elements, polys per element, bits per coefficient and HBM bytes held. */
XPIR_B200_API int xpir_b200_db_info(const xpir_b200_db *db, uint64_t *nb_aggregated, uint64_t *polys_per_element,
                      uint32_t *bits_per_coeff, uint64_t *device_bytes);
/* Copies the imported polys to host memory, in the reference's per-element layout
 * [element][poly][modulus][coefficient] (nb_aggregated * P * m * N words). */
XPIR_B200_API int xpir_b200_db_export(const xpir_b200_db *db, uint64_t *host_out, uint64_t capacity_words);

/* ---- reply ---------------------------------------------------------------------- */
/* Generates the reply of one query against an imported database: the level loop of
 * PIRReplyGeneratorNFL_internal::generateReply (…NFL_internal.cpp:340-445) with the
 * per-slot Shoup multiply-accumulate (crypto/NFLLWE.cpp:176-205) and the on-device
 * re-import of each level's replies as the next level's database (…NFL_internal.cpp:
 * 599-626).  `d` and `n` are PIRParameters.d and .n (pir/PIRParameters.hpp:24-29);
 * prod(n) must be at least the number of aggregated elements.  `query` holds sum(n)
 * ciphertexts (host memory if query_on_device == 0).  `replies` receives the final
 * ciphertexts (host memory if out_on_device == 0), `capacity_bytes` long; their count
 * is written to *nb_replies.  Replaces libpir's PIRReplyGenerator::generateReply
 * (pir/libpir.cpp:106-135); the outputs are what popReply hands out. */
XPIR_B200_API int xpir_b200_reply(xpir_b200_ctx *ctx, const xpir_b200_db *db, uint32_t d, const uint32_t *n, const void *query,
                    int query_on_device, void *replies, uint64_t capacity_bytes, int out_on_device,
                    uint64_t *nb_replies);

/* ---- batches of queries ---------------------------------------------------------- */
/* One query of a batch.  Query and reply buffers are device memory. */
typedef struct xpir_b200_request {
  const xpir_b200_db *db;            /* imported database the query is for */
  uint32_t d;                        /* PIRParameters.d */
  uint32_t n[XPIR_B200_MAX_LEVELS];  /* PIRParameters.n */
  const void *query;                 /* sum(n) ciphertexts, device memory */
  void *replies;                     /* device memory for the final ciphertexts */
  uint64_t capacity_bytes;
  int status;                        /* out: XPIR_B200_* for this query */
  uint64_t nb_replies;               /* out: reply ciphertexts written */
} xpir_b200_request;

/* Replies to `count` queries, possibly of different shapes and databases, in one
 * submission: queries that share a database and a shape run as one launch per
 * recursion level (the CTAs of all of them that read the same database tile run side
 * by side and share it through L2), and the d > 1 queries' level replies are
 * re-imported together.  Each reply is bit-identical to xpir_b200_reply's for the same
 * query.  With use_graph != 0 the launches are captured in a CUDA graph, cached by the
 * request list (databases, shapes and buffer addresses) and replayed when the same list
 * is submitted again.  No counterpart in the reference, which answers one query per
 * PIRReplyGenerator (pir/libpir.cpp:106-135); this is the batched form of that call.
 * Returns XPIR_B200_OK if every query succeeded (see each request's status). */
XPIR_B200_API int xpir_b200_reply_batch(xpir_b200_ctx *ctx, xpir_b200_request *reqs, uint32_t count, int use_graph);

/* Times the compiled tile shapes of the reply kernel on this query's level shapes
 * (queries in device memory; the replies are discarded) and keeps the fastest per
 * shape for later xpir_b200_reply / xpir_b200_reply_batch calls on this context.
 * *tile0 receives the choice for level 0.  No counterpart in the reference. */
XPIR_B200_API int xpir_b200_autotune(xpir_b200_ctx *ctx, const xpir_b200_db *db, uint32_t d, const uint32_t *n,
                                     const void *query_dev, int *tile0);

/* Pins the reply kernel's tile shape for one level shape (P polys per element, n_i slots
 * per group, `groups` groups) on this context, as xpir_b200_autotune keeps its choice;
 * tile -1 returns the shape to the default choice.  Tiles are numbered
 * 0 .. xpir_b200_tile_count()-1; one that cannot run the shape is refused with
 * XPIR_B200_ERR_ARG.  Replies do not depend on the tile.  No counterpart in the
 * reference. */
XPIR_B200_API int xpir_b200_set_level_tile(xpir_b200_ctx *ctx, uint64_t P, uint32_t n_i, uint64_t groups, int tile);
XPIR_B200_API int xpir_b200_tile_count(void);

/* ---- reply extraction (client side) ------------------------------------------------ */
/* Ciphertexts decrypted at recursion level `level` (1 = innermost) for an aggregated
 * element of aggregated_bytes (alpha * element bytes): the float arithmetic of
 * PIRReplyExtraction_internal::extractReply (pir/replyExtraction/PIRReplyExtraction_internal.cpp:50-58).
 * At level d this is the number of replies to pass to xpir_b200_extract. */
XPIR_B200_API uint64_t xpir_b200_extract_count(uint64_t aggregated_bytes, uint32_t level, uint32_t bits_per_coeff,
                                               uint32_t poly_degree, uint32_t nb_moduli);
/* Decrypts d-level replies with the client's secret key and recovers the aggregated
 * element: PIRReplyExtraction::extractReply + popPlaintextResult (pir/libpir.cpp:171-201,
 * PIRReplyExtraction_internal.cpp:41-106) with NFLLWE::decrypt (crypto/NFLLWE.cpp:375-475,
 * 515-551), on the GPU.  secret_key: host memory, [nb_moduli][poly_degree] u64 words in the
 * NTT domain, as NFLLWE keeps its secretKey.  replies: xpir_b200_extract_count(..., d, ...)
 * ciphertexts (host memory unless replies_on_device).  The first aggregated_bytes bytes
 * of the element are written to plaintext (host memory unless out_on_device).  Supports
 * up to 4 moduli (fewer than 128 bits per coefficient). */
XPIR_B200_API int xpir_b200_extract(xpir_b200_ctx *ctx, const uint64_t *secret_key, uint32_t d, uint32_t bits_per_coeff,
                                    uint64_t aggregated_bytes, const void *replies, uint64_t nb_replies,
                                    int replies_on_device, void *plaintext, uint64_t capacity_bytes,
                                    int out_on_device);

/* The client-side entry points (extraction and query generation) take their device
 * buffers (the key, host-side inputs or outputs staged on the device, the levels'
 * intermediates) from a stream-ordered pool of the context that keeps freed memory for
 * the next call; xpir_b200_ctx_destroy releases it. */

/* ---- query generation (client side) ------------------------------------------------ */
/* The sum(n) query ciphertexts of PIRQueryGenerator::generateQuery for chosen_element
 * (pir/queryGen/PIRQueryGenerator_internal.cpp:37-85), on the GPU: NFLLWE::encrypt of 1 at
 * each level's coordinate and of 0 elsewhere (crypto/NFLLWE.cpp:276-372, 481-498).  The
 * randomness is the reference's fastrandombytes stream (crypto/prng/fastrandombytes.cpp:34-55):
 * Salsa20/20 under the client's 32-byte prng_key, one nonce per PRNG call; ciphertext t
 * draws its noise with nonce first_nonce + 2t and its uniform half with first_nonce + 2t + 1
 * (for a fresh crypto object, key generation used nonce 0, so first_nonce = 1).
 * secret_key: host, [nb_moduli][poly_degree] words as NFLLWE's secretKey.  query receives
 * the ciphertexts back to back (host memory unless out_on_device).  No counterpart on the
 * reference's server path: the reference generates queries on the client's CPU. */
XPIR_B200_API int xpir_b200_generate_query(xpir_b200_ctx *ctx, const uint8_t *prng_key, uint64_t first_nonce,
                                           const uint64_t *secret_key, uint32_t d, const uint32_t *n,
                                           uint64_t chosen_element, uint32_t bits_per_coeff, uint32_t security_bits,
                                           void *query, uint64_t capacity_bytes, int out_on_device);

/* NFLLWE's secret key (crypto/NFLLWE.cpp:108-116): the uniform polynomial of the PRNG
 * call with the given nonce (0 for a fresh crypto object), written to host memory
 * ([nb_moduli][poly_degree] words, NTT domain). */
XPIR_B200_API int xpir_b200_generate_secret_key(xpir_b200_ctx *ctx, const uint8_t *prng_key, uint64_t nonce,
                                                uint64_t *secret_key);

/* ---- optimizer costs ------------------------------------------------------------------- */
/* The two per-plaintext costs XPIR's optimizer caches for a parameter set
 * (PIROptimizer::getAbs1PlaintextTime / getPrecompute1PlaintextTime,
 * pir/replyGenerator/PIROptimizer.cpp:155-209, with generateReplySimulation /
 * precomputationSimulation, PIRReplyGeneratorNFL_internal.cpp:446-498), measured on this
 * context's GPU: seconds of reply and of import per absorbed plaintext for a query over 4
 * elements, the element size doubled until a reply takes target_s seconds (<= 0: 0.05 s)
 * or the reference's 2^30-bit limit is reached. */
XPIR_B200_API int xpir_b200_measure_costs(xpir_b200_ctx *ctx, uint32_t security_bits, double target_s,
                                          double *reply_s_per_plaintext, double *import_s_per_plaintext);

/* ---- serving loop ------------------------------------------------------------------ */
/* A server over one or more contexts, one lane each.  Queries wait in FIFO order per
 * lane and are admitted while their device footprint (query, replies, recursion
 * workspace) fits what is left of `device_budget_bytes`; each lane runs the admitted
 * prefix (at most max_batch queries) as one xpir_b200_reply_batch, and queries that arrive
 * meanwhile join the next batch.  A lane is a two-stage pipeline (an uploading thread with
 * its own copy stream, a computing thread with the context's stream), so one batch's
 * host-to-device copies overlap the previous batch's replies, and lanes overlap each other.
 * No counterpart in the reference, whose server handles one query per session
 * (apps/server/PIRSession.cpp:45-111, 467-565). */
typedef struct xpir_b200_server xpir_b200_server;
XPIR_B200_API int xpir_b200_server_create(xpir_b200_server **srv, xpir_b200_ctx *const *ctxs, uint32_t nctx,
                                          uint64_t device_budget_bytes, uint32_t max_batch);
/* Queues one query (host buffers; both must stay valid until xpir_b200_server_wait for
 * the ticket returns).  XPIR_B200_ERR_NOMEM if its footprint exceeds the whole budget. */
XPIR_B200_API int xpir_b200_server_submit(xpir_b200_server *srv, const xpir_b200_db *db, uint32_t d, const uint32_t *n,
                                          const void *query, void *replies, uint64_t capacity_bytes, uint64_t *ticket);
/* Waits for a query (timeout_ms < 0: no limit) and returns its status; latency is from
 * submission to replies in host memory, queued_s from submission to admission.
 * XPIR_B200_ERR_STATE if the ticket is unknown or not done within the timeout. */
XPIR_B200_API int xpir_b200_server_wait(xpir_b200_server *srv, uint64_t ticket, int timeout_ms, uint64_t *nb_replies,
                                        double *latency_s, double *queued_s);
XPIR_B200_API int xpir_b200_server_stats(xpir_b200_server *srv, uint64_t *completed, uint64_t *batches,
                                         uint64_t *max_batch, uint64_t *peak_device_bytes);
/* Device bytes the server reserves while one query of this shape is admitted: its query
 * and reply buffers and its share of the recursion workspace (for sizing budgets). */
XPIR_B200_API int xpir_b200_server_footprint(const xpir_b200_db *db, uint32_t d, const uint32_t *n, uint64_t *bytes);
/* Stops the lanes: admitted queries run to completion, queries still waiting for
 * admission complete with XPIR_B200_ERR_STATE.  No xpir_b200_server_wait may be in
 * progress or follow; the server's contexts can then be destroyed. */
XPIR_B200_API int xpir_b200_server_destroy(xpir_b200_server *srv);

/* ---- reply without allocation ---------------------------------------------------- */
/* Bytes of device scratch available to xpir_b200_reply_noalloc (64 MiB). */
#define XPIR_B200_NOALLOC_SCRATCH_BYTES (64ull << 20)
/* No counterpart in the reference: an extra entry point of this library.
 *
 * Same result as xpir_b200_reply for a query and a reply buffer that are both already in
 * device memory, but this call allocates nothing: no cudaMalloc, cudaFree or pinned
 * buffer.  It is meant for callers that must not allocate while serving a request, for
 * example a caller that has set up all its memory in advance under a fixed device-memory
 * budget, or that runs inside an allocator or memory-pool hook of its own where a
 * nested allocation is not allowed.  The intermediate data of a recursive query (the
 * replies of each level and the next level's database) goes to one fixed scratch area
 * of XPIR_B200_NOALLOC_SCRATCH_BYTES that the library holds in the global memory of
 * every GPU that loads it, until the process exits.  A query whose intermediate data
 * does not fit is rejected with XPIR_B200_ERR_ARG before anything is launched; a d = 1
 * query uses no scratch.
 *
 * The set-up happens in xpir_b200_ctx_create, which (with the context's device current)
 * loads every engine kernel and the scratch area onto the device and looks up the scratch
 * area's device address with cudaGetSymbolAddress, so that no call here loads a module
 * (which would reserve device memory).  The context and the imported database are
 * created beforehand with the allocating calls above.  All calls share the one scratch
 * area and it keeps the previous call's contents (every word a call reads there is
 * written by the same call first): calls that overlap on the same GPU, from different
 * threads or contexts, race with each other and must be serialised by the caller.  The
 * caller's current device is the same after the call as before it. */
XPIR_B200_API int xpir_b200_reply_noalloc(xpir_b200_ctx *ctx, const xpir_b200_db *db, uint32_t d, const uint32_t *n,
                                          const void *query_dev, void *replies_dev, uint64_t capacity_bytes,
                                          uint64_t *nb_replies);

#ifdef __cplusplus
}
#endif

#endif /* XPIR_B200_H */
