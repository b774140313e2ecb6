/* The B200 engine as seen from inside XPIR: the pieces that XPIR's reply generators
 * share when they run on the GPU.  Compiled with XPIR's own headers, in XPIR's tree,
 * beside libpir_b200.cpp (libpir's PIRReplyGenerator) and PIRReplyGeneratorB200.cpp (the
 * server's GenericPIRReplyGenerator).
 *
 *   - one engine context per (GPU, poly degree, moduli) for the whole process, which
 *     holds the NTT tables on the device (the role of NFLlib::configureNTT,
 *     crypto/NFLlib.cpp:44-194, for the device);
 *   - ImportedDatabase, the object imported_database(_t)::imported_database_ptr points
 *     to when the engine imported the database (pir/replyGenerator/
 *     GenericPIRReplyGenerator.hpp:34-41): an engine database resident in HBM;
 *   - QueryBuffer, the query elements collected in push order (the role of queriesBuf,
 *     PIRReplyGeneratorNFL_internal.cpp:686-781, without the CPU Shoup factors: the
 *     engine derives them on the device);
 *   - import() and reply(), the engine's xpir_b200_db_import / xpir_b200_reply driven
 *     with XPIR's objects: the DBHandler streams and PIRParameters.
 *
 * Errors from the engine are thrown as b200::Error (a std::runtime_error naming the
 * engine status): XPIR's generator methods return nothing, and a reply that silently
 * stayed empty would leave popReply and the server's upload loop polling forever.
 * The GPU is taken from the environment variable XPIR_B200_DEVICE (default 0).
 */
#ifndef XPIR_B200_XPIR_ENGINE_HPP
#define XPIR_B200_XPIR_ENGINE_HPP

#include <stdint.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "crypto/LatticesBasedCryptosystem.hpp"
#include "pir/PIRParameters.hpp"
#include "pir/dbhandlers/DBHandler.hpp"
#include "xpir_b200.h"

namespace b200 {

struct Error : std::runtime_error {
  int status;
  Error(int status, const std::string &where);
};

// The engine context for this crypto object's parameter set on the configured GPU,
// created on first use and kept for the life of the process.
xpir_b200_ctx *context(LatticesBasedCryptosystem *crypto);

// Bits absorbed per coefficient as the crypto object is currently set
// (NFLLWE::setandgetAbsBitPerCiphertext, crypto/NFLLWE.cpp:656-668).
uint32_t bits_per_coeff(LatticesBasedCryptosystem *crypto);

// Bytes of one query or reply ciphertext (getCiphertextBitsize()/8).
uint64_t ciphertext_bytes(LatticesBasedCryptosystem *crypto);

// An imported database resident in HBM; deleting it frees the device copy.
struct ImportedDatabase {
  xpir_b200_db *db = nullptr;
  uint64_t element_bytes = 0;      // bytes of each element that were imported
  uint64_t nb_aggregated = 0;      // ceil(elements / alpha)
  uint64_t polys_per_element = 0;  // P
  uint32_t bits_per_coeff = 0;
  uint32_t alpha = 1;
  ~ImportedDatabase();
};

// Imports bytes [offset, offset + bytes_per_element) of every element of `db` (clipped
// to the longest element, zero-padded past each element's end by the handler), for
// queries of `params`: the work of PIRReplyGeneratorNFL_internal::importDataNFL
// (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:79-158).  The aggregation of
// DBHandler::readAggregatedStream (pir/dbhandlers/DBHandler.cpp:3-26), the bit split,
// the CRT and the NTT run on the GPU.
ImportedDatabase *import(LatticesBasedCryptosystem *crypto, DBHandler *db, const PIRParameters &params,
                         uint64_t offset, uint64_t bytes_per_element);

// The query elements of one PIR query, stored back to back in push order (level 0's
// n[0] elements first).  put() copies one element and frees the caller's buffer, which
// the generator owns from the push on (pushQuery takes ownership in XPIR).
class QueryBuffer {
 public:
  void reset(const PIRParameters &params, uint64_t ciphertext_bytes);
  void put(unsigned dim, unsigned nbr, char *raw, uint64_t size);
  // The next element in push order (libpir's pushQuery(char*)).
  void push(char *raw);
  bool ready() const { return total_ != 0; }
  bool complete() const { return pushed_ == total_ && total_ != 0; }
  const char *data() const { return bytes_.data(); }
  // Releases the stored elements; reset() must come before the next push.
  void clear();

 private:
  std::vector<char> bytes_;
  std::vector<uint64_t> level_start_;  // first element index of each level
  std::vector<unsigned> n_;
  std::vector<bool> have_;
  uint64_t ct_bytes_ = 0, total_ = 0, pushed_ = 0, next_ = 0;
};

// Generates the reply of a complete query against `db`: the level loop of
// PIRReplyGeneratorNFL_internal::generateReply (…NFL_internal.cpp:340-445) on the GPU.
// Returns the reply ciphertexts back to back (count = size / ciphertext_bytes).
std::vector<char> reply(LatticesBasedCryptosystem *crypto, const ImportedDatabase &db, const PIRParameters &params,
                        const QueryBuffer &query);

// Hands `replies` out as `count` malloc'd ciphertexts, publishing each one into
// slots[first + i] with a release store, as the NFL generator fills repliesArray
// (…NFL_internal.cpp:573) for popReply and the server's upload loop to poll.
void publish(char **slots, uint64_t first, const std::vector<char> &replies, uint64_t ct_bytes);

// A zeroed reply-pointer array of `count` entries, as generateReply allocates it (calloc:
// freed by the generator's freeResult with free()).
char **new_reply_array(uint64_t count);

}  // namespace b200

#endif
