// libpir with the B200 reply engine: the definitions of everything libpir.hpp declares,
// linked into XPIR's pir library in place of pir/libpir.cpp.  libpir.hpp itself is
// unchanged, so an application written against libpir (apps/simplepir/simplePIR.cpp)
// recompiles and relinks with no source change.
//
// Only the server side changes: PIRReplyGenerator (libpir.hpp:101-169) imports the
// database into HBM and generates the reply on the GPU through the engine's C ABI, with
// libpir's ownership rules (pushQuery takes each query element; popReply hands out
// malloc'd ciphertexts; deleting the imported_database frees the device copy).  The
// client classes (PIRQueryGenerator, PIRReplyExtraction) and the crypto factory forward
// to XPIR's internal classes exactly as the stock libpir does (pir/libpir.cpp:13-75,
// 165-213): queries, keys and extraction stay XPIR's own CPU code.
//
// libpir.hpp fixes PIRReplyGenerator's members, so the query the engine needs in one
// piece is kept in a table beside the generator, keyed by the generator's address; it is
// released by freeQueries() (simplePIR calls it before deleting the generator) and
// replaced when a new generator is constructed at the same address.
#include "libpir.hpp"

#include <stdlib.h>
#include <string.h>

#include <cmath>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <thread>

#include "b200_engine.hpp"

namespace {

std::mutex g_queries_mu;
std::map<const void *, std::unique_ptr<b200::QueryBuffer>> g_queries;

b200::QueryBuffer &query_of(const void *generator) {
  std::lock_guard<std::mutex> lock(g_queries_mu);
  std::unique_ptr<b200::QueryBuffer> &q = g_queries[generator];
  if (!q) q.reset(new b200::QueryBuffer());
  return *q;
}

void drop_query_of(const void *generator) {
  std::lock_guard<std::mutex> lock(g_queries_mu);
  g_queries.erase(generator);
}

}  // namespace

// ---- imported_database (libpir.hpp) ---------------------------------------------------

imported_database::~imported_database() {
  // The engine's database in HBM (b200::import); the stock destructor freed host polys.
  delete static_cast<b200::ImportedDatabase *>(imported_database_ptr);
  imported_database_ptr = NULL;
}

// ---- HomomorphicCryptoFactory -------------------------------------------------------

HomomorphicCrypto *HomomorphicCryptoFactory::getCryptoMethod(std::string cryptoType) {
  return HomomorphicCryptoFactory_internal::getCryptoMethod(cryptoType);
}

void HomomorphicCryptoFactory::printAllCryptoParams() {
  std::cout << "Available crypto parameters : (CryptoSystem::SecurityMax::PolyDegree::ModulusBitsize)"
            << std::endl;
  NFLLWE lwe;
  std::set<std::string> params;
  lwe.getAllCryptoParams(params);
  for (const std::string &p : params) std::cout << p << std::endl;
  std::cout << std::endl;
}

// ---- PIRQueryGenerator (client side, XPIR's code) ---------------------------------------

PIRQueryGenerator::PIRQueryGenerator(PIRParameters &pirParameters, HomomorphicCrypto &cryptoMethod_)
    : PIRQueryGenerator_internal(pirParameters, cryptoMethod_) {}

void PIRQueryGenerator::generateQuery(uint64_t _chosenElement) {
  nbQueries = 0;
  for (unsigned i = 0; i < pirParams.d; i++) nbQueries += pirParams.n[i];
  PIRQueryGenerator_internal::setChosenElement(_chosenElement);
  PIRQueryGenerator_internal::generateQuery();
}

bool PIRQueryGenerator::popQuery(char **query) {
  if (nbQueries == 0) return false;
  *query = queryBuffer.pop_front();
  nbQueries--;
  return true;
}

uint64_t PIRQueryGenerator::getQueryElementBytesize() {
  return cryptoMethod.getPublicParameters().getCiphertextBitsize() / 8;
}

// ---- PIRReplyGenerator (server side, on the GPU) ----------------------------------------

PIRReplyGenerator::PIRReplyGenerator(PIRParameters &param, HomomorphicCrypto &cryptoMethod_, DBHandler *db)
    : PIRReplyGeneratorNFL_internal(param, db), nbRepliesToHandle(0), nbRepliesGenerated(0), currentReply(0) {
  PIRReplyGeneratorNFL_internal::setCryptoMethod(&cryptoMethod_);
  // Sets the absorption for n[0] on the crypto object, as the stock constructor does.
  PIRReplyGeneratorNFL_internal::setPirParams(param);
  b200::QueryBuffer &q = query_of(this);
  q.clear();
  q.reset(pirParam, b200::ciphertext_bytes(cryptoMethod));
}

void PIRReplyGenerator::pushQuery(char *rawQuery) {
  b200::QueryBuffer &q = query_of(this);
  if (!q.ready()) q.reset(pirParam, b200::ciphertext_bytes(cryptoMethod));
  q.push(rawQuery);
}

imported_database *PIRReplyGenerator::importData(uint64_t offset, uint64_t bytes_per_db_element) {
  std::unique_ptr<b200::ImportedDatabase> db(
      b200::import(cryptoMethod, dbhandler, pirParam, offset, bytes_per_db_element));
  imported_database *out = new imported_database();
  // Same bookkeeping as the stock importData (pir/libpir.cpp:90-103).
  out->nbElements = ceil((float)dbhandler->getNbStream() / pirParam.alpha);
  out->polysPerElement = db->polys_per_element;
  out->beforeImportElementBytesize = bytes_per_db_element;
  out->imported_database_ptr = db.release();
  return out;
}

void PIRReplyGenerator::generateReply(const imported_database *database) {
  nbRepliesToHandle = nbRepliesGenerated = currentReply = 0;
  freeResult();
  const b200::ImportedDatabase *db = static_cast<const b200::ImportedDatabase *>(database->imported_database_ptr);
  if (!db) throw b200::Error(XPIR_B200_ERR_ARG, "generateReply: the database was not imported by this library");
  repliesAmount = computeReplySizeInChunks(database->beforeImportElementBytesize);
  // popReply may already be polling on another thread: it sees the array once its
  // pointer is published, and each ciphertext once its slot is.
  char **slots = b200::new_reply_array(repliesAmount);
  __atomic_store_n(&repliesArray, slots, __ATOMIC_RELEASE);
  nbRepliesToHandle = nbRepliesGenerated = repliesAmount;
  const std::vector<char> replies = b200::reply(cryptoMethod, *db, pirParam, query_of(this));
  const uint64_t ct = b200::ciphertext_bytes(cryptoMethod);
  if (replies.size() / ct != repliesAmount)
    throw b200::Error(XPIR_B200_ERR_STATE, "generateReply: reply count differs from computeReplySizeInChunks");
  b200::publish(repliesArray, 0, replies, ct);
}

void PIRReplyGenerator::freeQueries() {
  PIRReplyGeneratorNFL_internal::freeQueries();
  drop_query_of(this);
}

bool PIRReplyGenerator::popReply(char **reply) {
  if (nbRepliesToHandle == 0) return false;
  nbRepliesToHandle--;
  char **slots;
  while ((slots = __atomic_load_n(&repliesArray, __ATOMIC_ACQUIRE)) == NULL ||
         __atomic_load_n(&slots[currentReply], __ATOMIC_ACQUIRE) == NULL)
    std::this_thread::sleep_for(std::chrono::milliseconds(10));
  *reply = slots[currentReply];
  slots[currentReply++] = NULL;
  return true;
}

uint64_t PIRReplyGenerator::getnbRepliesGenerated() { return nbRepliesGenerated; }

uint64_t PIRReplyGenerator::getReplyElementBytesize() {
  return cryptoMethod->getPublicParameters().getCiphertextBitsize() / 8;
}

// ---- PIRReplyExtraction (client side, XPIR's code) ----------------------------------------

PIRReplyExtraction::PIRReplyExtraction(PIRParameters &pirParameters, HomomorphicCrypto &cryptoMethod_)
    : PIRReplyExtraction_internal(pirParameters, cryptoMethod_), clearChunks("clearChunks"), nbPlaintextReplies(0) {}

void PIRReplyExtraction::pushEncryptedReply(char *rawBytes) { repliesBuffer.push(rawBytes); }

void PIRReplyExtraction::extractReply(uint64_t maxFileBytesize) {
  PIRReplyExtraction_internal::extractReply(pirParams.alpha * maxFileBytesize, &clearChunks);
  nbPlaintextReplies = getnbPlaintextReplies(maxFileBytesize);
}

bool PIRReplyExtraction::popPlaintextResult(char **result) {
  if (nbPlaintextReplies == 0) return false;
  *result = clearChunks.pop_front();
  nbPlaintextReplies--;
  return true;
}

uint64_t PIRReplyExtraction::getPlaintextReplyBytesize() {
  return cryptoMethod.getPublicParameters().getAbsorptionBitsize(0) / GlobalConstant::kBitsPerByte;
}

uint64_t PIRReplyExtraction::getnbPlaintextReplies(uint64_t maxFileBytesize) {
  return ceil((float)maxFileBytesize * pirParams.alpha / getPlaintextReplyBytesize());
}
