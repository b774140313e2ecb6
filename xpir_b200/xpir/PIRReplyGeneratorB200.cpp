// PIRReplyGeneratorB200: XPIR's GenericPIRReplyGenerator on the B200 engine (see the
// header).
#include "PIRReplyGeneratorB200.hpp"

#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <iostream>
#include <memory>

#include "pir/dbhandlers/DBGenerator.hpp"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

uint64_t db_budget_bytes() {
  const char *env = getenv("XPIR_B200_DB_BUDGET_BYTES");
  return env && *env ? strtoull(env, nullptr, 10) : (64ull << 30);
}

}  // namespace

PIRReplyGeneratorB200::PIRReplyGeneratorB200() : GenericPIRReplyGenerator() {}

PIRReplyGeneratorB200::PIRReplyGeneratorB200(PIRParameters &param, DBHandler *db)
    : GenericPIRReplyGenerator(param, db) {}

PIRReplyGeneratorB200::~PIRReplyGeneratorB200() {
  freeQueries();
  freeResult();
  // The base class locks `mutex` at construction; leave it unlocked.
  mutex.try_lock();
  mutex.unlock();
}

void PIRReplyGeneratorB200::setCryptoMethod(CryptographicSystem *cm) {
  // Only the lattice cryptosystem has an NFL reply path.
  crypto_ = dynamic_cast<LatticesBasedCryptosystem *>(cm);
  if (!crypto_) throw b200::Error(XPIR_B200_ERR_ARG, "setCryptoMethod: not an LWE crypto object");
}

void PIRReplyGeneratorB200::setPirParams(PIRParameters &param) {
  freeQueries();
  GenericPIRReplyGenerator::setPirParams(param);
  if (crypto_) crypto_->setandgetAbsBitPerCiphertext(pirParam.n[0]);
  initQueriesBuffer();
}

void PIRReplyGeneratorB200::initQueriesBuffer() {
  if (!crypto_) throw b200::Error(XPIR_B200_ERR_STATE, "initQueriesBuffer: no crypto object set");
  query_.reset(pirParam, b200::ciphertext_bytes(crypto_));
}

void PIRReplyGeneratorB200::pushQuery(char *rawQuery, unsigned int size, int dim, int nbr) {
  if (!query_.ready()) initQueriesBuffer();
  query_.put((unsigned)dim, (unsigned)nbr, rawQuery, size);
}

void PIRReplyGeneratorB200::freeQueries() { query_.clear(); }

void PIRReplyGeneratorB200::freeResult() {
  if (!repliesArray) return;
  for (unsigned i = 0; i < repliesAmount; i++) {
    free(repliesArray[i]);
    repliesArray[i] = NULL;
  }
  free(repliesArray);
  repliesArray = NULL;
}

unsigned long PIRReplyGeneratorB200::computeReplySizeInChunks(unsigned long int maxFileBytesize) {
  // PIRReplyGeneratorNFL_internal::computeReplySizeInChunks (…NFL_internal.cpp:667-679).
  return (unsigned long)xpir_b200_reply_count(maxFileBytesize, pirParam.alpha, pirParam.d,
                                              b200::bits_per_coeff(crypto_), crypto_->getpolyDegree(),
                                              crypto_->getnbModuli());
}

// Bytes of each element per imported chunk: whole absorption units, as many as the
// device budget holds for every element (PIRReplyGeneratorNFL_internal.cpp:210-247 sizes
// its chunks the same way from host memory).
uint64_t PIRReplyGeneratorB200::chunk_bytes() const {
  const uint64_t longest = dbhandler->getmaxFileBytesize();
  if (pirParam.alpha != 1 || pirParam.d > 1) return longest;  // only d = 1, alpha = 1 chunks
  const uint64_t N = crypto_->getpolyDegree(), m = crypto_->getnbModuli();
  const uint64_t abs_bytes = N * b200::bits_per_coeff(crypto_) / 8;  // one poly's worth of element bytes
  const uint64_t poly_bytes = m * N * 8;
  const uint64_t per_element = db_budget_bytes() / std::max<uint64_t>(1, dbhandler->getNbStream());
  const uint64_t polys = std::max<uint64_t>(1, per_element / poly_bytes);
  return std::min(longest, polys * abs_bytes);
}

void PIRReplyGeneratorB200::reply_into_array(const b200::ImportedDatabase &db, uint64_t first) {
  const std::vector<char> replies = b200::reply(crypto_, db, pirParam, query_);
  const uint64_t ct = b200::ciphertext_bytes(crypto_);
  if (first + replies.size() / ct > repliesAmount)
    throw b200::Error(XPIR_B200_ERR_STATE, "generateReply: more replies than the reply array holds");
  b200::publish(repliesArray, first, replies, ct);
}

imported_database_t PIRReplyGeneratorB200::generateReplyGeneric(bool keep_imported_data) {
  if (!crypto_) throw b200::Error(XPIR_B200_ERR_STATE, "generateReplyGeneric: no crypto object set");
  imported_database_t kept;
  kept.imported_database_ptr = NULL;
  kept.nbElements = kept.polysPerElement = kept.beforeImportElementBytesize = 0;
  const uint64_t longest = dbhandler->getmaxFileBytesize();
  const uint64_t chunk = chunk_bytes();
  const uint64_t iterations = (longest + chunk - 1) / chunk;
  if (iterations > 1) {
    keep_imported_data = false;  // a database that is not resident in one piece cannot be kept
    std::cout << "PIRReplyGeneratorB200: database larger than the device budget, processing it in " << iterations
              << " chunks" << std::endl;
  }
  const double start = now_s();
  freeResult();
  repliesAmount = computeReplySizeInChunks(longest);
  char **slots = b200::new_reply_array(repliesAmount);
  __atomic_store_n(&repliesArray, slots, __ATOMIC_RELEASE);
  for (uint64_t it = 0; it < iterations; it++) {
    // Chunk `it` is whole absorption units, so its replies are the full reply's from
    // computeReplySizeInChunks(it * chunk) on.
    repliesIndex = computeReplySizeInChunks(it * chunk);
    std::unique_ptr<b200::ImportedDatabase> db(b200::import(crypto_, dbhandler, pirParam, it * chunk, chunk));
    // The query may still be arriving (the session's download thread holds the lock until
    // the last element is pushed); the import above overlapped it.
    boost::mutex::scoped_lock lock(mutex);
    reply_into_array(*db, repliesIndex);
    if (keep_imported_data) {
      kept.polysPerElement = db->polys_per_element;
      kept.beforeImportElementBytesize = longest;
      kept.nbElements = dbhandler->getNbStream();
      kept.imported_database_ptr = (void *)db.release();
    }
  }
  std::cout << "PIRReplyGeneratorB200: total process time " << now_s() - start << " seconds" << std::endl;
  freeQueries();
  return kept;
}

void PIRReplyGeneratorB200::generateReplyGenericFromData(const imported_database_t database) {
  if (!crypto_) throw b200::Error(XPIR_B200_ERR_STATE, "generateReplyGenericFromData: no crypto object set");
  const b200::ImportedDatabase *db = (const b200::ImportedDatabase *)database.imported_database_ptr;
  if (!db) throw b200::Error(XPIR_B200_ERR_ARG, "generateReplyGenericFromData: no imported database");
  boost::mutex::scoped_lock lock(mutex);
  const double start = now_s();
  freeResult();
  repliesAmount = computeReplySizeInChunks(database.beforeImportElementBytesize);
  repliesIndex = 0;
  char **slots = b200::new_reply_array(repliesAmount);
  __atomic_store_n(&repliesArray, slots, __ATOMIC_RELEASE);
  reply_into_array(*db, 0);
  std::cout << "PIRReplyGeneratorB200: total process time " << now_s() - start << " seconds" << std::endl;
  freeQueries();
}

// The optimizer's reply-cost probe: prod(n) fake elements of plaintext_nbr plaintexts
// each, imported into HBM, and the wall time of one reply to an all-zero query (the
// timing does not depend on the words).  Same experiment as
// PIRReplyGeneratorNFL_internal::generateReplySimulation (…NFL_internal.cpp:446-466).
double PIRReplyGeneratorB200::generateReplySimulation(const PIRParameters &pir_params, uint64_t plaintext_nbr) {
  setPirParams((PIRParameters &)pir_params);
  uint64_t files = 1;
  for (unsigned i = 0; i < pirParam.d; i++) files *= pirParam.n[i];
  const uint64_t plain_bytes = (uint64_t)crypto_->getpolyDegree() * crypto_->getnbModuli() * 8;
  DBGenerator fake(files, plaintext_nbr * plain_bytes, true);
  std::unique_ptr<b200::ImportedDatabase> db(b200::import(crypto_, &fake, pirParam, 0, plaintext_nbr * plain_bytes));
  const uint64_t ct = b200::ciphertext_bytes(crypto_);
  uint64_t elements = 0;
  for (unsigned i = 0; i < pirParam.d; i++) elements += pirParam.n[i];
  for (uint64_t e = 0; e < elements; e++) query_.push((char *)calloc(ct, 1));
  const double start = now_s();
  (void)b200::reply(crypto_, *db, pirParam, query_);
  const double took = now_s() - start;
  freeQueries();
  return took;
}

// The optimizer's import-cost probe (…NFL_internal.cpp:470-498): the wall time of
// importing the same fake database into HBM.
double PIRReplyGeneratorB200::precomputationSimulation(const PIRParameters &pir_params, uint64_t plaintext_nbr) {
  setPirParams((PIRParameters &)pir_params);
  uint64_t files = 1;
  for (unsigned i = 0; i < pirParam.d; i++) files *= pirParam.n[i];
  const uint64_t plain_bytes = (uint64_t)crypto_->getpolyDegree() * crypto_->getnbModuli() * 8;
  DBGenerator fake(files, plaintext_nbr * plain_bytes, true);
  const double start = now_s();
  std::unique_ptr<b200::ImportedDatabase> db(b200::import(crypto_, &fake, pirParam, 0, plaintext_nbr * plain_bytes));
  const double took = now_s() - start;
  freeQueries();
  return took;
}
