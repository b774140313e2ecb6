// xpir_b200_pir.hpp -- C++ API of the B200 reply engine, shaped like XPIR's libpir
// (libpir.hpp:101-210, pir/libpir.cpp:77-201) so that a server written against libpir's
// PIRReplyGenerator (or a client using its PIRReplyExtraction) moves over by changing its
// includes and namespace.
//
// The classes sit on the C ABI of include/xpir_b200.h.  Semantics kept from libpir:
//   * pushQuery takes ownership of a malloc'd query ciphertext (freed by freeQueries);
//   * importData(offset, bytes) imports bytes [offset, offset+bytes) of every element,
//     aggregated alpha at a time, and returns an imported_database that owns the
//     database's device memory (freed by its destructor);
//   * generateReply computes the whole reply; popReply then hands out one malloc'd
//     ciphertext per call (the caller frees it) and returns false at the end;
//   * generateReplyGeneric is the memory-chunked import+reply of the reference's server
//     (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:202-292), chunked here by a
//     device-memory budget instead of half the host memory.
// Differences: errors (which libpir reports by printing, or by exiting on an invalid
// modulus) raise xpir_b200::Error carrying the engine's status; only the "LWE"
// cryptosystem exists; the database handler interface is the subset the reply side uses.
#ifndef XPIR_B200_PIR_HPP
#define XPIR_B200_PIR_HPP

#include <stdint.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "xpir_b200.h"

namespace xpir_b200 {

// An engine status other than XPIR_B200_OK.
class Error : public std::runtime_error {
 public:
  Error(int status, const std::string &where);
  int status;
};

// pir/PIRParameters.hpp:24-29.
constexpr unsigned MAX_REC_LVL = XPIR_B200_MAX_LEVELS;
struct PIRParameters {
  unsigned int alpha = 1;
  unsigned int d = 1;
  unsigned int n[MAX_REC_LVL] = {};
  std::string crypto_params;  // "LWE:<security bits>:<poly degree>:<60 * moduli>"
};

// The part of NFLLWE (crypto/NFLLWE.cpp) the reply side needs: the parameter set and the
// absorption size.  Created by HomomorphicCryptoFactory::getCryptoMethod.
class HomomorphicCrypto {
 public:
  HomomorphicCrypto(unsigned security_bits, unsigned poly_degree, unsigned nb_moduli);
  // NFLLWE::setandgetAbsBitPerCiphertext (crypto/NFLLWE.cpp:656-668): bits absorbed per
  // coefficient for a first dimension of n0 elements; kept for importData.
  unsigned setandgetAbsBitPerCiphertext(uint64_t n0);
  unsigned getAbsBitPerCiphertext() const { return abs_bits_; }
  unsigned getpolyDegree() const { return poly_degree_; }
  unsigned getnbModuli() const { return nb_moduli_; }
  unsigned getSecurityBits() const { return security_bits_; }
  uint64_t getCiphertextBytesize() const;  // getCiphertextBitsize()/8

 private:
  unsigned security_bits_, poly_degree_, nb_moduli_, abs_bits_ = 0;
};

// HomomorphicCryptoFactory::getCryptoMethod (pir/libpir.cpp:19-22) for "LWE:k:N:logq".
class HomomorphicCryptoFactory {
 public:
  static HomomorphicCrypto *getCryptoMethod(const std::string &crypto_params);
};

// The database handler interface of pir/dbhandlers/DBHandler.hpp:26-45 that the reply
// side calls: element count and size, and reads of an element from an offset (a short
// element reads as zeros past its end, as DBVectorProcessor::readStream does).
class DBHandler {
 public:
  virtual ~DBHandler() = default;
  virtual uint64_t getNbStream() = 0;
  virtual uint64_t getmaxFileBytesize() = 0;
  virtual bool openStream(uint64_t streamNb, uint64_t requested_offset) = 0;
  virtual uint64_t readStream(uint64_t streamNb, char *buf, uint64_t size) = 0;
  virtual void closeStream(uint64_t streamNb) = 0;
};

// Elements held in host memory (the role of pir/dbhandlers/DBVectorProcessor.cpp).
class DBVectorProcessor : public DBHandler {
 public:
  struct element_t {
    std::string name;
    std::vector<char> data;
  };
  explicit DBVectorProcessor(std::vector<element_t> elements);
  uint64_t getNbStream() override { return elements_.size(); }
  uint64_t getmaxFileBytesize() override { return max_bytes_; }
  bool openStream(uint64_t streamNb, uint64_t requested_offset) override;
  uint64_t readStream(uint64_t streamNb, char *buf, uint64_t size) override;
  void closeStream(uint64_t streamNb) override;

 private:
  std::vector<element_t> elements_;
  std::vector<uint64_t> pos_;
  uint64_t max_bytes_ = 0;
};

// The imported database (libpir's imported_database / imported_database_t,
// pir/replyGenerator/GenericPIRReplyGenerator.hpp:34-41): its polys live in HBM and are
// freed by the destructor (pir/libpir.cpp:5-11).
class imported_database {
 public:
  ~imported_database();
  imported_database(const imported_database &) = delete;
  imported_database &operator=(const imported_database &) = delete;
  uint64_t nbElements = 0;       // aggregated elements
  uint64_t polysPerElement = 0;
  uint64_t beforeImportElementBytesize = 0;
  xpir_b200_db *handle = nullptr;

 private:
  friend class PIRReplyGenerator;
  imported_database() = default;
  std::shared_ptr<xpir_b200_ctx> ctx_;  // keeps the parameter set alive
};

// libpir's PIRReplyGenerator (libpir.hpp:101-169) on a B200.
class PIRReplyGenerator {
 public:
  // device: the CUDA device of the engine context.
  PIRReplyGenerator(PIRParameters &param, HomomorphicCrypto &cryptoMethod, DBHandler *db, int device = 0);
  ~PIRReplyGenerator();

  // One query ciphertext (getReplyElementBytesize() bytes, malloc'd); the generator
  // owns it until freeQueries.  Ciphertexts come in PIRQueryGenerator's order: the
  // n[0] of the first dimension, then n[1], ...
  void pushQuery(char *rawQuery);
  // Bytes [offset, offset+bytes_per_db_element) of every element (bytes_per_db_element
  // WITHOUT the alpha factor, as in libpir), aggregated and imported into HBM.
  imported_database *importData(uint64_t offset, uint64_t bytes_per_db_element);
  // The reply of the pushed query against `database` (all levels).
  void generateReply(const imported_database *database);
  // The memory-chunked import+reply of the reference server for d = 1 and alpha = 1:
  // the elements' bytes are imported and answered in chunks that fit the device budget
  // (a multiple of the absorption size, so the replies are those of one full import).
  // With keep_imported_data and a single chunk the imported database is returned (the
  // caller deletes it); otherwise nullptr.  Other shapes run as one chunk.
  imported_database *generateReplyGeneric(bool keep_imported_data);
  // generateReplyGenericFromData (…NFL_internal.cpp:297-334): reply from a kept database.
  void generateReplyGenericFromData(const imported_database *database) { generateReply(database); }
  void freeQueries();
  // Hands out the next reply ciphertext (malloc'd; the caller frees it); false at the end.
  bool popReply(char **reply);
  uint64_t getnbRepliesGenerated() const { return nb_replies_; }
  uint64_t getReplyElementBytesize() const { return crypto_.getCiphertextBytesize(); }
  // Device bytes generateReplyGeneric may give one chunk's imported polys (default 16 GiB).
  void setDeviceMemoryBudget(uint64_t bytes) { budget_ = bytes; }

 private:
  imported_database *import_range(uint64_t offset, uint64_t bytes);
  void reply_into(const imported_database *database, uint64_t first_reply);

  PIRParameters param_;
  HomomorphicCrypto &crypto_;
  DBHandler *dbhandler_;
  std::shared_ptr<xpir_b200_ctx> ctx_;
  std::vector<char *> queries_;
  std::vector<uint64_t> replies_;  // nb_replies_ ciphertexts, contiguous
  uint64_t nb_replies_ = 0, next_reply_ = 0, budget_ = 0;
};

// libpir's PIRReplyExtraction (libpir.hpp:176-210, pir/libpir.cpp:165-201), client side,
// decrypting on the GPU with the client's secret key ([nb_moduli][poly_degree] words in
// the NTT domain, as XPIR's NFLLWE holds it).
class PIRReplyExtraction {
 public:
  PIRReplyExtraction(PIRParameters &param, HomomorphicCrypto &cryptoMethod, std::vector<uint64_t> secret_key,
                     int device = 0);
  ~PIRReplyExtraction();
  // One reply ciphertext (malloc'd; the extractor owns it).
  void pushEncryptedReply(char *rawBytes);
  // Decrypts the pushed replies down to the element of maxFileBytesize bytes (times alpha).
  void extractReply(uint64_t maxFileBytesize);
  // The next plaintext chunk of getPlaintextReplyBytesize() bytes (malloc'd; the caller
  // frees it); false after getnbPlaintextReplies chunks.  The bytes past the aggregated
  // element in the last chunk read as zeros.
  bool popPlaintextResult(char **result);
  uint64_t getPlaintextReplyBytesize() const;
  uint64_t getnbPlaintextReplies(uint64_t maxFileBytesize) const;

 private:
  PIRParameters param_;
  HomomorphicCrypto &crypto_;
  std::vector<uint64_t> key_;
  std::shared_ptr<xpir_b200_ctx> ctx_;
  std::vector<char *> replies_;
  std::vector<char> plain_;
  uint64_t chunks_ = 0, next_ = 0;
};

}  // namespace xpir_b200

#endif
