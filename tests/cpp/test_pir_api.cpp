// The libpir-shaped C++ API (include/xpir_b200_pir.hpp) driven the way a libpir server
// drives PIRReplyGenerator (apps/simplepir/simplePIR.cpp:32-110): crypto object from its
// parameter string, absorption size from n[0], queries pushed one malloc'd ciphertext at
// a time, importData, generateReply, popReply until false.
//
//   test_pir_api params <crypto> <n0> <want_bits> <want_ct_bytes>
//       host-only checks (no GPU needed): parameter parsing, sizes, errors;
//   test_pir_api run <dir>
//       reads <dir>/params.txt ("crypto alpha d n0 .. n{d-1} budget"), <dir>/sizes.bin
//       (u64 per element: its byte length), <dir>/db.bin (the elements back to back) and
//       <dir>/query.bin; writes <dir>/reply.bin (generateReply) and
//       <dir>/reply_generic.bin (generateReplyGeneric under the given device budget);
//       with <dir>/key.bin present, PIRReplyExtraction decrypts the reply with that key
//       into <dir>/plain.bin (popPlaintextResult chunks, concatenated).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <fstream>
#include <iostream>
#include <iterator>
#include <memory>
#include <string>
#include <vector>

#include "xpir_b200_pir.hpp"

using namespace xpir_b200;

namespace {

std::vector<char> slurp(const std::string &path) {
  std::ifstream f(path, std::ios::binary);
  return std::vector<char>(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
}

bool spill(const std::string &path, const std::vector<char> &data) {
  std::ofstream f(path, std::ios::binary);
  f.write(data.data(), (std::streamsize)data.size());
  return (bool)f;
}

#define CHECK(c)                                          \
  do {                                                    \
    if (!(c)) {                                           \
      printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c); \
      return 1;                                           \
    }                                                     \
  } while (0)

int params_mode(char **argv) {
  std::unique_ptr<HomomorphicCrypto> crypto(HomomorphicCryptoFactory::getCryptoMethod(argv[2]));
  CHECK(crypto->setandgetAbsBitPerCiphertext(strtoull(argv[3], nullptr, 10)) == strtoul(argv[4], nullptr, 10));
  CHECK(crypto->getCiphertextBytesize() == strtoull(argv[5], nullptr, 10));
  for (const char *bad : {"Paillier:1024:2048", "LWE:80:2048", "LWE:80:2048:100", "LWE:x:2048:120"}) {
    bool threw = false;
    try {
      delete HomomorphicCryptoFactory::getCryptoMethod(bad);
    } catch (const Error &e) {
      threw = e.status == XPIR_B200_ERR_ARG;
    }
    CHECK(threw);
  }
  // Without a usable GPU the generator reports it instead of falling back.
  DBVectorProcessor db({{"a", std::vector<char>(100, 1)}});
  PIRParameters p;
  p.n[0] = 1;
  int count = 0;
  xpir_b200_device_count(&count);
  if (count == 0) {
    bool threw = false;
    try {
      PIRReplyGenerator g(p, *crypto, &db);
    } catch (const Error &e) {
      threw = e.status == XPIR_B200_ERR_NODEV;
    }
    CHECK(threw);
  }
  // The in-memory handler reads zeros past a short element's end.
  DBVectorProcessor v({{"x", {1, 2, 3}}, {"y", {4, 5, 6, 7, 8}}});
  CHECK(v.getNbStream() == 2 && v.getmaxFileBytesize() == 5);
  char buf[5];
  CHECK(v.openStream(0, 1));
  v.readStream(0, buf, 4);
  v.closeStream(0);
  CHECK(buf[0] == 2 && buf[1] == 3 && buf[2] == 0 && buf[3] == 0);
  printf("ok params\n");
  return 0;
}

int run_mode(const std::string &dir) {
  std::ifstream pf(dir + "/params.txt");
  PIRParameters params;
  uint64_t budget = 0;
  pf >> params.crypto_params >> params.alpha >> params.d;
  for (unsigned i = 0; i < params.d; i++) pf >> params.n[i];
  pf >> budget;
  CHECK((bool)pf);
  const std::vector<char> sizes = slurp(dir + "/sizes.bin"), bytes = slurp(dir + "/db.bin");
  const std::vector<char> query = slurp(dir + "/query.bin");
  const uint64_t nb = sizes.size() / 8;
  std::vector<DBVectorProcessor::element_t> elements(nb);
  uint64_t at = 0;
  for (uint64_t i = 0; i < nb; i++) {
    uint64_t len;
    memcpy(&len, sizes.data() + 8 * i, 8);
    elements[i].name = std::to_string(i);
    elements[i].data.assign(bytes.begin() + at, bytes.begin() + at + len);
    at += len;
  }
  DBVectorProcessor db(std::move(elements));

  std::unique_ptr<HomomorphicCrypto> crypto(HomomorphicCryptoFactory::getCryptoMethod(params.crypto_params));
  crypto->setandgetAbsBitPerCiphertext(params.n[0]);
  const uint64_t ct = crypto->getCiphertextBytesize();
  uint64_t nq = 0;
  for (unsigned i = 0; i < params.d; i++) nq += params.n[i];
  CHECK(query.size() == nq * ct);
  auto push_all = [&](PIRReplyGenerator &g) {
    for (uint64_t i = 0; i < nq; i++) {
      char *q = (char *)malloc(ct);  // ownership passes to the generator
      memcpy(q, query.data() + i * ct, ct);
      g.pushQuery(q);
    }
  };
  auto pop_all = [&](PIRReplyGenerator &g) {
    std::vector<char> out;
    char *r;
    while (g.popReply(&r)) {
      out.insert(out.end(), r, r + g.getReplyElementBytesize());
      free(r);
    }
    return out;
  };

  PIRReplyGenerator gen(params, *crypto, &db);
  CHECK(gen.getReplyElementBytesize() == ct);
  push_all(gen);
  std::unique_ptr<imported_database> imported(gen.importData(0, db.getmaxFileBytesize()));
  gen.generateReply(imported.get());
  const uint64_t count = gen.getnbRepliesGenerated();
  std::vector<char> reply = pop_all(gen);
  CHECK(reply.size() == count * ct);
  // The same imported database answers a second query (libpir's reuse pattern).
  gen.freeQueries();
  push_all(gen);
  gen.generateReply(imported.get());
  CHECK(pop_all(gen) == reply);
  CHECK(spill(dir + "/reply.bin", reply));

  PIRReplyGenerator gen2(params, *crypto, &db);
  gen2.setDeviceMemoryBudget(budget);
  push_all(gen2);
  std::unique_ptr<imported_database> kept(gen2.generateReplyGeneric(true));
  std::vector<char> generic = pop_all(gen2);
  CHECK(generic.size() == gen2.getnbRepliesGenerated() * ct);
  CHECK(spill(dir + "/reply_generic.bin", generic));
  const std::vector<char> keybytes = slurp(dir + "/key.bin");
  if (!keybytes.empty()) {
    std::vector<uint64_t> key(keybytes.size() / 8);
    memcpy(key.data(), keybytes.data(), key.size() * 8);
    PIRReplyExtraction ex(params, *crypto, key);
    for (uint64_t i = 0; i * ct < reply.size(); i++) {
      char *r = (char *)malloc(ct);  // ownership passes to the extractor
      memcpy(r, reply.data() + i * ct, ct);
      ex.pushEncryptedReply(r);
    }
    ex.extractReply(db.getmaxFileBytesize());
    std::vector<char> plain;
    char *chunk;
    uint64_t chunks = 0;
    while (ex.popPlaintextResult(&chunk)) {
      plain.insert(plain.end(), chunk, chunk + ex.getPlaintextReplyBytesize());
      free(chunk);
      chunks++;
    }
    CHECK(chunks == ex.getnbPlaintextReplies(db.getmaxFileBytesize()));
    CHECK(spill(dir + "/plain.bin", plain));
  }
  printf("ok run replies=%llu generic=%llu kept=%d\n", (unsigned long long)count,
         (unsigned long long)gen2.getnbRepliesGenerated(), kept ? 1 : 0);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  try {
    if (argc >= 6 && !strcmp(argv[1], "params")) return params_mode(argv);
    if (argc >= 3 && !strcmp(argv[1], "run")) return run_mode(argv[2]);
  } catch (const std::exception &e) {
    printf("FAIL exception: %s\n", e.what());
    return 1;
  }
  fprintf(stderr, "usage: test_pir_api params <crypto> <n0> <bits> <ct_bytes> | run <dir>\n");
  return 2;
}
