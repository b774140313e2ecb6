// C++ server-side API shaped like XPIR's libpir (see include/xpir_b200_pir.hpp), on top
// of the engine's C ABI.  Host code only: it stages database bytes, keeps the pushed
// query and the generated replies in host memory, and calls xpir_b200_* for everything
// that runs on the GPU.
#include "xpir_b200_pir.hpp"

#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <iostream>
#include <sstream>

namespace xpir_b200 {

namespace {

std::string describe(int status, const std::string &where) {
  std::ostringstream os;
  os << where << ": " << xpir_b200_strerror(status) << " (status " << status
     << ", last CUDA error " << xpir_b200_last_cuda_error() << ")";
  return os.str();
}

void check(int status, const char *where) {
  if (status != XPIR_B200_OK) throw Error(status, where);
}

}  // namespace

Error::Error(int s, const std::string &where) : std::runtime_error(describe(s, where)), status(s) {}

// ---- crypto parameters -------------------------------------------------------------

HomomorphicCrypto::HomomorphicCrypto(unsigned security_bits, unsigned poly_degree, unsigned nb_moduli)
    : security_bits_(security_bits), poly_degree_(poly_degree), nb_moduli_(nb_moduli) {
  if (xpir_b200_ciphertext_bytes(poly_degree, nb_moduli) == 0)
    throw Error(XPIR_B200_ERR_ARG, "HomomorphicCrypto: unsupported poly degree or modulus count");
}

unsigned HomomorphicCrypto::setandgetAbsBitPerCiphertext(uint64_t n0) {
  const int32_t b = xpir_b200_bits_per_coeff(poly_degree_, nb_moduli_, security_bits_, n0);
  if (b <= 0) throw Error(XPIR_B200_ERR_ARG, "setandgetAbsBitPerCiphertext: no bits left to absorb");
  abs_bits_ = (unsigned)b;
  return abs_bits_;
}

uint64_t HomomorphicCrypto::getCiphertextBytesize() const {
  return xpir_b200_ciphertext_bytes(poly_degree_, nb_moduli_);
}

// "LWE:<security>:<degree>:<modulus bits>", the parameter string of
// NFLLWE::setNewParameters (crypto/NFLLWE.cpp:55-120); the modulus is a product of
// 60-bit primes, so its size is a multiple of 60.
HomomorphicCrypto *HomomorphicCryptoFactory::getCryptoMethod(const std::string &crypto_params) {
  std::vector<std::string> f;
  std::stringstream ss(crypto_params);
  for (std::string item; std::getline(ss, item, ':');) f.push_back(item);
  if (f.size() < 4 || f[0] != "LWE")
    throw Error(XPIR_B200_ERR_ARG, "getCryptoMethod: expected LWE:<security>:<degree>:<modulus bits>, got " +
                                       crypto_params);
  unsigned long k, N, logq;
  try {
    k = std::stoul(f[1]);
    N = std::stoul(f[2]);
    logq = std::stoul(f[3]);
  } catch (const std::exception &) {
    throw Error(XPIR_B200_ERR_ARG, "getCryptoMethod: malformed parameters " + crypto_params);
  }
  if (logq == 0 || logq % 60 != 0)
    throw Error(XPIR_B200_ERR_ARG, "getCryptoMethod: modulus size must be a multiple of 60 bits");
  return new HomomorphicCrypto((unsigned)k, (unsigned)N, (unsigned)(logq / 60));
}

// ---- in-memory database --------------------------------------------------------------

DBVectorProcessor::DBVectorProcessor(std::vector<element_t> elements)
    : elements_(std::move(elements)), pos_(elements_.size(), ~0ull) {
  for (const element_t &e : elements_) max_bytes_ = std::max<uint64_t>(max_bytes_, e.data.size());
}

bool DBVectorProcessor::openStream(uint64_t streamNb, uint64_t requested_offset) {
  if (streamNb >= elements_.size() || pos_[streamNb] != ~0ull) return false;
  pos_[streamNb] = requested_offset;
  return true;
}

uint64_t DBVectorProcessor::readStream(uint64_t streamNb, char *buf, uint64_t size) {
  const std::vector<char> &d = elements_[streamNb].data;
  const uint64_t at = pos_[streamNb];
  const uint64_t have = at < d.size() ? std::min<uint64_t>(size, d.size() - at) : 0;
  if (have) memcpy(buf, d.data() + at, have);
  if (have < size) memset(buf + have, 0, size - have);
  pos_[streamNb] = at + size;
  return size;
}

void DBVectorProcessor::closeStream(uint64_t streamNb) {
  if (streamNb < pos_.size()) pos_[streamNb] = ~0ull;
}

// ---- imported database ---------------------------------------------------------------

imported_database::~imported_database() {
  if (handle) xpir_b200_db_free(handle);
}

// ---- reply generator -----------------------------------------------------------------

PIRReplyGenerator::PIRReplyGenerator(PIRParameters &param, HomomorphicCrypto &cryptoMethod, DBHandler *db,
                                     int device)
    : param_(param), crypto_(cryptoMethod), dbhandler_(db) {
  if (!db) throw Error(XPIR_B200_ERR_ARG, "PIRReplyGenerator: no database handler");
  if (param.d == 0 || param.d > MAX_REC_LVL || param.alpha == 0)
    throw Error(XPIR_B200_ERR_ARG, "PIRReplyGenerator: invalid PIR parameters");
  xpir_b200_ctx *ctx = nullptr;
  check(xpir_b200_ctx_create(&ctx, device, crypto_.getpolyDegree(), crypto_.getnbModuli()),
        "PIRReplyGenerator: context");
  ctx_.reset(ctx, [](xpir_b200_ctx *c) { xpir_b200_ctx_destroy(c); });
  budget_ = 16ull << 30;
}

PIRReplyGenerator::~PIRReplyGenerator() { freeQueries(); }

void PIRReplyGenerator::pushQuery(char *rawQuery) {
  if (!rawQuery) throw Error(XPIR_B200_ERR_ARG, "pushQuery: null query");
  queries_.push_back(rawQuery);
}

void PIRReplyGenerator::freeQueries() {
  for (char *q : queries_) free(q);
  queries_.clear();
}

imported_database *PIRReplyGenerator::import_range(uint64_t offset, uint64_t bytes) {
  const uint64_t nb = dbhandler_->getNbStream(), L = dbhandler_->getmaxFileBytesize();
  if (nb == 0 || offset >= L || bytes == 0) throw Error(XPIR_B200_ERR_ARG, "importData: empty range");
  const uint64_t len = std::min(bytes, L - offset);  // readAggregatedStream's fileByteSize
  if (crypto_.getAbsBitPerCiphertext() == 0) crypto_.setandgetAbsBitPerCiphertext(param_.n[0]);
  // Each element's range, zero-filled past its end; the aggregation (including the
  // reference's handling of a short last group) happens on the device.
  std::vector<char> staged(nb * len);
  for (uint64_t i = 0; i < nb; i++) {
    dbhandler_->openStream(i, offset);
    dbhandler_->readStream(i, staged.data() + i * len, len);
    dbhandler_->closeStream(i);
  }
  std::unique_ptr<imported_database> out(new imported_database());
  out->ctx_ = ctx_;
  check(xpir_b200_db_import(ctx_.get(), staged.data(), nb, len, len, param_.alpha, crypto_.getAbsBitPerCiphertext(),
                            0, &out->handle),
        "importData");
  uint64_t nagg = 0, P = 0, dev_bytes = 0;
  uint32_t b = 0;
  check(xpir_b200_db_info(out->handle, &nagg, &P, &b, &dev_bytes), "importData: info");
  out->nbElements = nagg;
  out->polysPerElement = P;
  out->beforeImportElementBytesize = bytes;
  return out.release();
}

imported_database *PIRReplyGenerator::importData(uint64_t offset, uint64_t bytes_per_db_element) {
  return import_range(offset, bytes_per_db_element);
}

void PIRReplyGenerator::reply_into(const imported_database *database, uint64_t first_reply) {
  uint64_t nq = 0;
  for (unsigned i = 0; i < param_.d; i++) nq += param_.n[i];
  if (queries_.size() != nq) throw Error(XPIR_B200_ERR_STATE, "generateReply: incomplete query");
  const uint64_t ct = crypto_.getCiphertextBytesize();
  std::vector<char> query(nq * ct);
  for (uint64_t i = 0; i < nq; i++) memcpy(query.data() + i * ct, queries_[i], ct);
  const uint64_t words = ct / 8;
  const uint64_t cap = (nb_replies_ - first_reply) * ct;
  uint64_t count = 0;
  check(xpir_b200_reply(ctx_.get(), database->handle, param_.d, param_.n, query.data(), 0,
                        replies_.data() + first_reply * words, cap, 0, &count),
        "generateReply");
}

void PIRReplyGenerator::generateReply(const imported_database *database) {
  if (!database || !database->handle) throw Error(XPIR_B200_ERR_ARG, "generateReply: no database");
  // Reply count of the reference (computeReplySizeInChunks of the imported size).
  nb_replies_ = xpir_b200_reply_count(database->beforeImportElementBytesize, param_.alpha, param_.d,
                                      crypto_.getAbsBitPerCiphertext(), crypto_.getpolyDegree(),
                                      crypto_.getnbModuli());
  next_reply_ = 0;
  replies_.assign(nb_replies_ * (crypto_.getCiphertextBytesize() / 8), 0);
  reply_into(database, 0);
}

imported_database *PIRReplyGenerator::generateReplyGeneric(bool keep_imported_data) {
  const uint64_t nb = dbhandler_->getNbStream(), L = dbhandler_->getmaxFileBytesize();
  if (crypto_.getAbsBitPerCiphertext() == 0) crypto_.setandgetAbsBitPerCiphertext(param_.n[0]);
  const uint64_t N = crypto_.getpolyDegree(), m = crypto_.getnbModuli(), b = crypto_.getAbsBitPerCiphertext();
  const uint64_t abs_bytes = b * N / 8;  // bytes absorbed by one poly (N is a multiple of 8)
  // Polys per element that fit the budget, then the chunk as whole absorption units
  // (…NFL_internal.cpp:222-226), at least one unit and at most the element.
  const uint64_t per_poly = (uint64_t)std::max<uint64_t>(1, (nb + param_.alpha - 1) / param_.alpha) * m * N * 8;
  uint64_t chunk = std::max<uint64_t>(1, budget_ / per_poly) * abs_bytes;
  chunk = std::min(chunk, L);
  uint64_t iterations = (L + chunk - 1) / chunk;
  if (iterations > 1 && (param_.alpha != 1 || param_.d > 1)) {
    std::cerr << "PIRReplyGenerator: aggregation or recursion cannot be chunked; importing the database at once"
              << std::endl;
    chunk = L;
    iterations = 1;
  }
  nb_replies_ = xpir_b200_reply_count(L, param_.alpha, param_.d, (uint32_t)b, (uint32_t)N, (uint32_t)m);
  next_reply_ = 0;
  replies_.assign(nb_replies_ * (crypto_.getCiphertextBytesize() / 8), 0);
  imported_database *kept = nullptr;
  for (uint64_t it = 0; it < iterations; it++) {
    const uint64_t offset = it * chunk;
    std::unique_ptr<imported_database> db(import_range(offset, chunk));
    db->beforeImportElementBytesize = iterations == 1 ? L : chunk;
    // A chunk starts on an absorption boundary, so its polys are the full import's polys
    // offset / abs_bytes and on (computeReplySizeInChunks(offset), …NFL_internal.cpp:254).
    reply_into(db.get(), offset / abs_bytes);
    if (keep_imported_data && iterations == 1) kept = db.release();
  }
  freeQueries();
  return kept;
}

bool PIRReplyGenerator::popReply(char **reply) {
  if (!reply || next_reply_ >= nb_replies_) return false;
  const uint64_t ct = crypto_.getCiphertextBytesize();
  char *out = (char *)malloc(ct);
  if (!out) throw Error(XPIR_B200_ERR_NOMEM, "popReply");
  memcpy(out, (const char *)replies_.data() + next_reply_ * ct, ct);
  next_reply_++;
  *reply = out;
  return true;
}

// ---- reply extraction ------------------------------------------------------------------

PIRReplyExtraction::PIRReplyExtraction(PIRParameters &param, HomomorphicCrypto &cryptoMethod,
                                       std::vector<uint64_t> secret_key, int device)
    : param_(param), crypto_(cryptoMethod), key_(std::move(secret_key)) {
  if ((uint64_t)key_.size() != (uint64_t)crypto_.getnbModuli() * crypto_.getpolyDegree())
    throw Error(XPIR_B200_ERR_ARG, "PIRReplyExtraction: the key needs nb_moduli * poly_degree words");
  xpir_b200_ctx *ctx = nullptr;
  check(xpir_b200_ctx_create(&ctx, device, crypto_.getpolyDegree(), crypto_.getnbModuli()),
        "PIRReplyExtraction: context");
  ctx_.reset(ctx, [](xpir_b200_ctx *c) { xpir_b200_ctx_destroy(c); });
}

PIRReplyExtraction::~PIRReplyExtraction() {
  for (char *r : replies_) free(r);
}

void PIRReplyExtraction::pushEncryptedReply(char *rawBytes) {
  if (!rawBytes) throw Error(XPIR_B200_ERR_ARG, "pushEncryptedReply: null reply");
  replies_.push_back(rawBytes);
}

uint64_t PIRReplyExtraction::getPlaintextReplyBytesize() const {
  return (uint64_t)crypto_.getAbsBitPerCiphertext() * crypto_.getpolyDegree() / 8;
}

uint64_t PIRReplyExtraction::getnbPlaintextReplies(uint64_t maxFileBytesize) const {
  // libpir.cpp:196-198
  return (uint64_t)std::ceil((float)maxFileBytesize * param_.alpha / (float)getPlaintextReplyBytesize());
}

void PIRReplyExtraction::extractReply(uint64_t maxFileBytesize) {
  if (crypto_.getAbsBitPerCiphertext() == 0) crypto_.setandgetAbsBitPerCiphertext(param_.n[0]);
  const uint64_t agg = maxFileBytesize * param_.alpha, ct = crypto_.getCiphertextBytesize();
  const uint32_t b = crypto_.getAbsBitPerCiphertext();
  const uint64_t need = xpir_b200_extract_count(agg, param_.d, b, crypto_.getpolyDegree(), crypto_.getnbModuli());
  if (replies_.size() < need) throw Error(XPIR_B200_ERR_STATE, "extractReply: fewer replies than the element needs");
  std::vector<char> replies(need * ct);
  for (uint64_t i = 0; i < need; i++) memcpy(replies.data() + i * ct, replies_[i], ct);
  chunks_ = getnbPlaintextReplies(maxFileBytesize);
  plain_.assign(chunks_ * getPlaintextReplyBytesize(), 0);
  check(xpir_b200_extract(ctx_.get(), key_.data(), param_.d, b, agg, replies.data(), need, 0, plain_.data(),
                          plain_.size(), 0),
        "extractReply");
  next_ = 0;
  for (char *r : replies_) free(r);
  replies_.clear();
}

bool PIRReplyExtraction::popPlaintextResult(char **result) {
  if (!result || next_ >= chunks_) return false;
  const uint64_t pb = getPlaintextReplyBytesize();
  char *out = (char *)malloc(pb);
  if (!out) throw Error(XPIR_B200_ERR_NOMEM, "popPlaintextResult");
  memcpy(out, plain_.data() + next_ * pb, pb);
  next_++;
  *result = out;
  return true;
}

}  // namespace xpir_b200
