/* PIRReplyGeneratorB200 -- XPIR's NFLLWE reply generator on a B200 GPU, compiled inside
 * XPIR with XPIR's headers, and returned by PIRReplyGeneratorFactory for "LWE" in place
 * of PIRReplyGeneratorNFL_internal (pir/replyGenerator/PIRReplyGeneratorFactory.cpp:20-43).
 *
 * It implements the GenericPIRReplyGenerator interface that XPIR's server drives
 * (pir/replyGenerator/GenericPIRReplyGenerator.hpp:44-73; apps/server/PIRSession.cpp:
 * 389-565, PIRServer.cpp:71-104):
 *   initQueriesBuffer, pushQuery(buf, size, dim, nbr)   the query elements as the session
 *                                                       downloads them (the generator
 *                                                       takes ownership of each buffer);
 *   generateReplyGeneric(keep)                          imports the database into HBM (in
 *                                                       chunks when it exceeds the device
 *                                                       budget), waits on `mutex` for the
 *                                                       whole query, replies; with keep the
 *                                                       imported database is returned for
 *                                                       later sessions (driven mode);
 *   generateReplyGenericFromData(db)                    replies from such a kept database;
 *   computeReplySizeInChunks                            as the NFL generator.
 * Each reply ciphertext is published into repliesArray as a malloc'd buffer that the
 * consumer (PIRSession::uploadWorker, libpir's popReply) frees, as the NFL generator does.
 * The replies are bit-identical to PIRReplyGeneratorNFL_internal's.
 *
 * generateReplySimulation / precomputationSimulation (the optimizer's cost probes,
 * PIRReplyGeneratorNFL_internal.cpp:446-498) run the same fake-data experiment on the GPU.
 *
 * The device budget for one imported chunk is XPIR_B200_DB_BUDGET_BYTES (default 64 GiB);
 * like the NFL generator, only d = 1, alpha = 1 databases are chunked.
 */
#ifndef DEF_PIRREPLYGENERATORB200
#define DEF_PIRREPLYGENERATORB200

#include <stdint.h>

#include "b200_engine.hpp"
#include "crypto/LatticesBasedCryptosystem.hpp"
#include "pir/replyGenerator/GenericPIRReplyGenerator.hpp"

class PIRReplyGeneratorB200 : public GenericPIRReplyGenerator {
 public:
  PIRReplyGeneratorB200();
  PIRReplyGeneratorB200(PIRParameters &param, DBHandler *db);
  ~PIRReplyGeneratorB200();

  void setCryptoMethod(CryptographicSystem *cm);
  void initQueriesBuffer();
  void pushQuery(char *rawQuery, unsigned int size, int dim, int nbr);
  imported_database_t generateReplyGeneric(bool keep_imported_data = false);
  void generateReplyGenericFromData(const imported_database_t database);
  double generateReplySimulation(const PIRParameters &pir_params, uint64_t plaintext_nbr);
  double precomputationSimulation(const PIRParameters &pir_params, uint64_t plaintext_nbr);
  unsigned long computeReplySizeInChunks(unsigned long int maxFileBytesize);

  // The PIR parameters, with the crypto object's absorption set for n[0] (as
  // PIRReplyGeneratorNFL_internal::setPirParams, …NFL_internal.cpp:804-811).
  void setPirParams(PIRParameters &param);
  void freeQueries();
  void freeResult();

 private:
  void reply_into_array(const b200::ImportedDatabase &db, uint64_t first);
  uint64_t chunk_bytes() const;

  LatticesBasedCryptosystem *crypto_ = nullptr;
  b200::QueryBuffer query_;
};

#endif
