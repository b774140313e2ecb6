// PIRReplyGeneratorFactory with the B200 engine: linked into XPIR's pir library in place
// of pir/replyGenerator/PIRReplyGeneratorFactory.cpp (declarations unchanged in
// PIRReplyGeneratorFactory.hpp).  "LWE" now yields PIRReplyGeneratorB200, so the server
// (apps/server/PIRSession.cpp:230) and the optimizer (pir/replyGenerator/PIROptimizer.cpp:
// 104-209) reply and measure on the GPU; the other cryptosystems keep XPIR's generators.
#include "pir/replyGenerator/PIRReplyGeneratorFactory.hpp"

#include <iostream>

#include "PIRReplyGeneratorB200.hpp"

GenericPIRReplyGenerator *PIRReplyGeneratorFactory::getPIRReplyGenerator(const std::string &gen_name,
                                                                         PIRParameters &param, DBHandler *db) {
  if (gen_name == "LWE") return new PIRReplyGeneratorB200(param, db);
  if (gen_name == "Paillier") return new PIRReplyGeneratorGMP(param, db);
  if (gen_name == "NoCryptography") return new PIRReplyGeneratorTrivial(param, db);
  std::cout << "PIRReplyGeneratorFactory: Could not find an appropriate generator for " << gen_name
            << ", returning NULL" << std::endl;
  return NULL;
}

GenericPIRReplyGenerator *PIRReplyGeneratorFactory::getPIRReplyGenerator(const std::string &gen_name) {
  if (gen_name == "LWE") return new PIRReplyGeneratorB200();
  if (gen_name == "Paillier") return new PIRReplyGeneratorGMP();
  std::cout << "PIRReplyGeneratorFactory (optim function): Could not find an appropriate generator for "
            << gen_name << ", returning NULL" << std::endl;
  return NULL;
}
