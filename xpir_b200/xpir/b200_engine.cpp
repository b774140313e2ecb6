// The B200 engine as seen from inside XPIR (see b200_engine.hpp).
#include "b200_engine.hpp"

#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <sstream>
#include <tuple>

namespace b200 {

namespace {

std::string describe(int status, const std::string &where) {
  std::ostringstream os;
  os << "B200 reply engine: " << where << ": " << xpir_b200_strerror(status) << " (status " << status
     << ", last CUDA error " << xpir_b200_last_cuda_error() << ")";
  return os.str();
}

void check(int status, const char *where) {
  if (status != XPIR_B200_OK) throw Error(status, where);
}

int configured_device() {
  const char *env = getenv("XPIR_B200_DEVICE");
  return env && *env ? atoi(env) : 0;
}

}  // namespace

Error::Error(int s, const std::string &where) : std::runtime_error(describe(s, where)), status(s) {}

xpir_b200_ctx *context(LatticesBasedCryptosystem *crypto) {
  // Contexts are never destroyed: imported databases kept by a server (driven mode)
  // outlive the generator that made them, and a context owns its databases.
  static std::mutex mu;
  static std::map<std::tuple<int, unsigned, unsigned>, xpir_b200_ctx *> contexts;
  const int device = configured_device();
  const unsigned N = crypto->getpolyDegree(), m = crypto->getnbModuli();
  std::lock_guard<std::mutex> lock(mu);
  xpir_b200_ctx *&ctx = contexts[std::make_tuple(device, N, m)];
  if (!ctx) check(xpir_b200_ctx_create(&ctx, device, N, m), "context");
  return ctx;
}

uint32_t bits_per_coeff(LatticesBasedCryptosystem *crypto) {
  return crypto->getPublicParameters().getAbsorptionBitsize(0) / crypto->getpolyDegree();
}

uint64_t ciphertext_bytes(LatticesBasedCryptosystem *crypto) {
  return crypto->getPublicParameters().getCiphertextBitsize() / 8;
}

ImportedDatabase::~ImportedDatabase() {
  if (db) xpir_b200_db_free(db);
}

ImportedDatabase *import(LatticesBasedCryptosystem *crypto, DBHandler *dbh, const PIRParameters &params,
                         uint64_t offset, uint64_t bytes_per_element) {
  if (!crypto || !dbh) throw Error(XPIR_B200_ERR_ARG, "import: no crypto object or database handler");
  const uint64_t nb = dbh->getNbStream(), longest = dbh->getmaxFileBytesize();
  if (nb == 0 || offset >= longest || bytes_per_element == 0)
    throw Error(XPIR_B200_ERR_ARG, "import: empty database range");
  // readAggregatedStream's fileByteSize: the range clipped to the longest element.
  const uint64_t len = std::min(bytes_per_element, longest - offset);
  const uint32_t b = bits_per_coeff(crypto);
  if (b == 0) throw Error(XPIR_B200_ERR_ARG, "import: the crypto object absorbs no bits (set n[0] first)");
  // Every element's range, zero-padded by the handler past the element's end; grouping
  // by alpha (and the reference's short-last-group behaviour) happens on the device.
  std::vector<char> staged(nb * len);
  for (uint64_t i = 0; i < nb; i++) {
    dbh->openStream(i, offset);
    dbh->readStream(i, staged.data() + i * len, len);
    dbh->closeStream(i);
  }
  xpir_b200_ctx *ctx = context(crypto);
  ImportedDatabase *out = new ImportedDatabase();
  out->element_bytes = len;
  out->alpha = params.alpha;
  out->bits_per_coeff = b;
  const int rc = xpir_b200_db_import(ctx, staged.data(), nb, len, len, params.alpha, b, 0, &out->db);
  if (rc != XPIR_B200_OK) {
    delete out;
    throw Error(rc, "import");
  }
  uint32_t bits = 0;
  check(xpir_b200_db_info(out->db, &out->nb_aggregated, &out->polys_per_element, &bits, nullptr), "import");
  return out;
}

void QueryBuffer::reset(const PIRParameters &params, uint64_t ct_bytes) {
  ct_bytes_ = ct_bytes;
  n_.assign(params.n, params.n + params.d);
  level_start_.assign(params.d, 0);
  total_ = 0;
  for (unsigned i = 0; i < params.d; i++) {
    level_start_[i] = total_;
    total_ += params.n[i];
  }
  bytes_.assign(total_ * ct_bytes_, 0);
  have_.assign(total_, false);
  pushed_ = next_ = 0;
}

void QueryBuffer::put(unsigned dim, unsigned nbr, char *raw, uint64_t size) {
  if (!raw) throw Error(XPIR_B200_ERR_ARG, "pushQuery: null query element");
  if (!ready()) {
    free(raw);
    throw Error(XPIR_B200_ERR_STATE, "pushQuery: the query buffer is not set up");
  }
  if (dim >= n_.size() || nbr >= n_[dim] || size < ct_bytes_) {
    free(raw);
    throw Error(XPIR_B200_ERR_ARG, "pushQuery: element outside the query's dimensions");
  }
  const uint64_t at = level_start_[dim] + nbr;
  memcpy(bytes_.data() + at * ct_bytes_, raw, ct_bytes_);
  free(raw);
  if (!have_[at]) {
    have_[at] = true;
    pushed_++;
  }
}

void QueryBuffer::push(char *raw) {
  if (next_ >= total_) {
    free(raw);
    throw Error(XPIR_B200_ERR_STATE, "pushQuery: more elements than the query has");
  }
  unsigned dim = 0;
  while (dim + 1 < level_start_.size() && next_ >= level_start_[dim + 1]) dim++;
  put(dim, (unsigned)(next_ - level_start_[dim]), raw, ct_bytes_);
  next_++;
}

void QueryBuffer::clear() {
  std::vector<char>().swap(bytes_);
  std::vector<bool>().swap(have_);
  n_.clear();
  level_start_.clear();
  total_ = pushed_ = next_ = 0;
}

std::vector<char> reply(LatticesBasedCryptosystem *crypto, const ImportedDatabase &db, const PIRParameters &params,
                        const QueryBuffer &query) {
  if (!query.complete()) throw Error(XPIR_B200_ERR_STATE, "generateReply: the query is incomplete");
  if (db.bits_per_coeff != bits_per_coeff(crypto) || db.alpha != params.alpha)
    throw Error(XPIR_B200_ERR_ARG, "generateReply: the database was imported for other PIR parameters");
  const uint64_t ct = ciphertext_bytes(crypto);
  const uint64_t count = xpir_b200_reply_count(db.element_bytes, params.alpha, params.d, db.bits_per_coeff,
                                               crypto->getpolyDegree(), crypto->getnbModuli());
  std::vector<char> out(count * ct);
  uint64_t written = 0;
  check(xpir_b200_reply(context(crypto), db.db, params.d, params.n, query.data(), 0, out.data(), out.size(), 0,
                        &written),
        "reply");
  if (written != count) throw Error(XPIR_B200_ERR_STATE, "reply: unexpected number of ciphertexts");
  return out;
}

void publish(char **slots, uint64_t first, const std::vector<char> &replies, uint64_t ct_bytes) {
  const uint64_t count = replies.size() / ct_bytes;
  for (uint64_t i = 0; i < count; i++) {
    char *r = (char *)malloc(ct_bytes);
    if (!r) throw Error(XPIR_B200_ERR_NOMEM, "publish: out of host memory");
    memcpy(r, replies.data() + i * ct_bytes, ct_bytes);
    __atomic_store_n(&slots[first + i], r, __ATOMIC_RELEASE);
  }
}

char **new_reply_array(uint64_t count) {
  char **a = (char **)calloc(count ? count : 1, sizeof(char *));
  if (!a) throw Error(XPIR_B200_ERR_NOMEM, "reply array: out of host memory");
  return a;
}

}  // namespace b200
