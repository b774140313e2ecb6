// The nine cases of XPIR's apps/simplepir/simplePIR.cpp (:212-344), on seeded data,
// driven through XPIR's own classes.  Test infrastructure: compiled twice against XPIR's
// sources, once with the stock libpir and reply-generator factory (the reference,
// oracle/_ref/xpir_simplepir) and once with the B200 ones (libpir_b200.cpp,
// PIRReplyGeneratorFactory_b200.cpp), so that the replies of the two builds can be
// compared byte for byte.
//
//   xpir_simplepir libpir <case> <dir>   the simplePIR flow (simplePIR.cpp:3-182):
//       HomomorphicCryptoFactory -> PIRQueryGenerator -> PIRReplyGenerator::pushQuery,
//       importData, generateReply, popReply -> PIRReplyExtraction.
//   xpir_simplepir server <case> <dir>   the server's flow (apps/server/PIRSession.cpp:
//       215-240, 383-565, PIRServer.cpp:71-104): a crypto object rebuilt from the client's
//       serialized parameters, a generator from PIRReplyGeneratorFactory("LWE"), the
//       query pushed element by element from a download thread that then unlocks the
//       generator's mutex, replies taken from repliesArray by an upload thread; a first
//       session keeps the imported database (driven mode) and a second session, with a
//       new generator and a new query, replies from it with generateReplyGenericFromData.
//
// <dir> receives replies.bin (and replies2.bin for the second server session); stdout
// gets one JSON line with the element recovered by XPIR's PIRReplyExtraction.
// Databases: DBVectorProcessor over seeded bytes of the sizes simplePIR uses (its
// DBGenerator cases), and DBDirectoryProcessor over seeded files written to <dir>/db/
// for cases 6 and 7.  Keys and queries come from XPIR's PRNG with a seeded randombytes.
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "libpir.hpp"
#include "pir/replyGenerator/PIRReplyGeneratorFactory.hpp"

#include <pthread.h>

extern "C" void xpir_ref_set_seed(uint64_t seed);

namespace {

int g_result_fd = 1;

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

uint64_t g_rng = 1;
unsigned char next_byte() {
  g_rng ^= g_rng << 13;
  g_rng ^= g_rng >> 7;
  g_rng ^= g_rng << 17;
  return (unsigned char)(g_rng >> 24);
}

std::vector<char> seeded_bytes(uint64_t n) {
  std::vector<char> v(n);
  for (uint64_t i = 0; i < n; i++) v[i] = (char)next_byte();
  return v;
}

void write_file(const std::string &path, const std::vector<char> &data) {
  FILE *f = fopen(path.c_str(), "wb");
  if (!f || fwrite(data.data(), 1, data.size(), f) != data.size()) {
    fprintf(stderr, "xpir_simplepir: cannot write %s\n", path.c_str());
    exit(2);
  }
  fclose(f);
}

// One simplePIR case: the database handler and the PIR parameters.
struct Case {
  DBHandler *db = nullptr;
  std::vector<element_t> elements;  // backing store of a DBVectorProcessor
  PIRParameters params;
  uint64_t chosen = 0, chosen2 = 0;
};

void set_params(Case &c, unsigned alpha, std::vector<unsigned> n) {
  c.params.alpha = alpha;
  c.params.d = (unsigned)n.size();
  for (int i = 0; i < MAX_REC_LVL; i++) c.params.n[i] = i < (int)n.size() ? n[i] : 0;
  c.params.crypto_params = "LWE:80:2048:120";
}

void vector_db(Case &c, const std::vector<uint64_t> &sizes) {
  for (size_t i = 0; i < sizes.size(); i++) {
    std::vector<char> bytes = seeded_bytes(sizes[i]);
    char *data = (char *)malloc(sizes[i]);
    memcpy(data, bytes.data(), sizes[i]);
    c.elements.push_back(Element("element" + std::to_string(i), sizes[i], data));
  }
  c.db = new DBVectorProcessor(c.elements);
}

// simplePIR's cases 1-9 (simplePIR.cpp:212-344) with seeded contents.  Cases 8 and 9
// keep n[0] from case 7, as simplePIR's reused PIRParameters do.
Case make_case(int k, const std::string &dir) {
  Case c;
  g_rng = 0x9E3779B97F4A7C15ull ^ (uint64_t)k * 0x2545F4914F6CDD1Dull;
  const uint64_t big = 1ull << 25;
  const std::vector<uint64_t> dir7_sizes = {4096, 70000, 1, 33333, 12288, 65536};
  switch (k) {
    case 1: set_params(c, 1, {20}); vector_db(c, std::vector<uint64_t>(20, (1ull << 20) / 20)); c.chosen = 3; c.chosen2 = 17; break;
    case 2: set_params(c, 100, {1}); vector_db(c, std::vector<uint64_t>(100, big / 100)); c.chosen = 0; c.chosen2 = 0; break;
    case 3: set_params(c, 1, {50, 2}); vector_db(c, std::vector<uint64_t>(100, big / 100)); c.chosen = 3; c.chosen2 = 77; break;
    case 4: set_params(c, 2, {25, 2}); vector_db(c, std::vector<uint64_t>(100, big / 100)); c.chosen = 3; c.chosen2 = 41; break;
    case 5: set_params(c, 1, {5, 5, 4}); vector_db(c, std::vector<uint64_t>(100, big / 100)); c.chosen = 3; c.chosen2 = 99; break;
    case 6: {
      // DBDirectoryProcessor(4) splits the directory's first file into 4 streams.
      mkdir((dir + "/db").c_str(), 0755);
      write_file(dir + "/db/file0", seeded_bytes(big));
      set_params(c, 1, {4});
      c.db = new DBDirectoryProcessor(4);
      c.chosen = 3;
      c.chosen2 = 1;
      break;
    }
    case 7: {
      mkdir((dir + "/db").c_str(), 0755);
      for (size_t i = 0; i < dir7_sizes.size(); i++)
        write_file(dir + "/db/file" + std::to_string(i), seeded_bytes(dir7_sizes[i]));
      c.db = new DBDirectoryProcessor();
      set_params(c, 1, {(unsigned)c.db->getNbStream()});
      c.chosen = 0;
      c.chosen2 = 4;
      break;
    }
    case 8: set_params(c, 1, {(unsigned)dir7_sizes.size()}); vector_db(c, {10, 11, 8}); c.chosen = 0; c.chosen2 = 2; break;
    case 9: set_params(c, 2, {(unsigned)dir7_sizes.size()}); vector_db(c, {10, 11, 8, 14, 13}); c.chosen = 0; c.chosen2 = 1; break;
    default: fprintf(stderr, "xpir_simplepir: case %d does not exist\n", k); exit(2);
  }
  return c;
}

// The client side of simplePIR: crypto object, query, and the check of the recovered
// element (simplePIR.cpp:12-31, 121-166).
struct Client {
  HomomorphicCrypto *crypto;
  PIRParameters params;
  explicit Client(const PIRParameters &p) : params(p) {
    crypto = HomomorphicCryptoFactory::getCryptoMethod(params.crypto_params);
    crypto->setandgetAbsBitPerCiphertext(params.n[0]);
  }
  ~Client() { delete crypto; }
  std::vector<char *> query(uint64_t chosen) {
    PIRQueryGenerator q(params, *crypto);
    q.generateQuery(chosen);
    std::vector<char *> out;
    char *e;
    while (q.popQuery(&e)) out.push_back(e);
    return out;
  }
  // Decrypts the replies (taking them) and compares with the chosen aggregated element.
  bool extract(DBHandler *db, const std::vector<char *> &replies, uint64_t chosen) {
    PIRReplyExtraction x(params, *crypto);
    for (char *r : replies) x.pushEncryptedReply(r);
    const uint64_t L = db->getmaxFileBytesize();
    x.extractReply(L);
    const uint64_t pb = x.getPlaintextReplyBytesize();
    std::vector<char> plain(x.getnbPlaintextReplies(L) * pb + pb);
    char *out = plain.data(), *tmp;
    while (x.popPlaintextResult(&tmp)) {
      memcpy(out, tmp, pb);
      out += pb;
      free(tmp);
    }
    std::vector<char> want(L * params.alpha);
    db->readAggregatedStream(chosen, params.alpha, 0, L, want.data());
    return memcmp(plain.data(), want.data(), want.size()) == 0;
  }
};

std::vector<char> concat(const std::vector<char *> &replies, uint64_t ct) {
  std::vector<char> all(replies.size() * ct);
  for (size_t i = 0; i < replies.size(); i++) memcpy(all.data() + i * ct, replies[i], ct);
  return all;
}

int run_libpir(Case &c, const std::string &dir) {
  Client client(c.params);
  std::vector<char *> q = client.query(c.chosen);
  PIRReplyGenerator *gen = new PIRReplyGenerator(c.params, *client.crypto, c.db);
  for (char *e : q) gen->pushQuery(e);
  double t0 = now_s();
  imported_database *imported = gen->importData(0, c.db->getmaxFileBytesize());
  const double import_s = now_s() - t0;
  t0 = now_s();
  gen->generateReply(imported);
  const double reply_s = now_s() - t0;
  std::vector<char *> replies;
  char *r;
  while (gen->popReply(&r)) replies.push_back(r);
  const uint64_t ct = gen->getReplyElementBytesize();
  write_file(dir + "/replies.bin", concat(replies, ct));
  const bool ok = client.extract(c.db, replies, c.chosen);
  dprintf(g_result_fd, "{\"mode\": \"libpir\", \"replies\": %zu, \"nb_generated\": %llu, \"import_s\": %.4f, \"reply_s\": %.4f, "
         "\"extract_ok\": %d}\n",
         replies.size(), (unsigned long long)gen->getnbRepliesGenerated(), import_s, reply_s, ok ? 1 : 0);
  delete imported;
  gen->freeQueries();
  delete gen;
  return ok ? 0 : 1;
}

// ---- server flow --------------------------------------------------------------------

struct Session {
  GenericPIRReplyGenerator *gen;
  HomomorphicCrypto *crypto;
  PIRParameters *params;
  std::vector<char *> query;
  uint64_t ct_bytes;
  unsigned long reply_nbr;
  std::vector<char *> replies;
};

// PIRSession::downloadWorker (PIRSession.cpp:383-459): one buffer per query element,
// pushed with its level and index, then the generator's mutex is unlocked.
void *download(void *arg) {
  Session *s = (Session *)arg;
  s->gen->initQueriesBuffer();
  size_t k = 0;
  for (unsigned j = 0; j < s->params->d; j++) {
    const unsigned msg = s->crypto->getPublicParameters().getQuerySizeFromRecLvl(j + 1) / 8;
    for (unsigned i = 0; i < s->params->n[j]; i++) {
      char *buf = (char *)malloc(msg);
      memcpy(buf, s->query[k], msg);
      free(s->query[k++]);
      s->gen->pushQuery(buf, msg, (int)j, (int)i);
    }
  }
  s->gen->mutex.unlock();
  return nullptr;
}

// PIRSession::uploadWorker (PIRSession.cpp:509-565): waits for each reply slot, takes it.
void *upload(void *arg) {
  Session *s = (Session *)arg;
  for (unsigned long i = 0; i < s->reply_nbr; i++) {
    char **slots;
    while ((slots = __atomic_load_n(&s->gen->repliesArray, __ATOMIC_ACQUIRE)) == NULL ||
           __atomic_load_n(&slots[i], __ATOMIC_ACQUIRE) == NULL)
      usleep(1000);
    char *ct = (char *)malloc(s->ct_bytes);
    memcpy(ct, slots[i], s->ct_bytes);
    free(slots[i]);
    slots[i] = NULL;
    s->replies.push_back(ct);
  }
  return nullptr;
}

int run_server(Case &c, const std::string &dir) {
  Client client(c.params);
  // The server's crypto object, rebuilt from the client's parameters (PIRSession.cpp:215-226).
  const std::string serialized = client.crypto->getSerializedCryptoParams(false);
  HomomorphicCrypto *server_crypto = HomomorphicCryptoFactory_internal::getCrypto("LWE");
  server_crypto->setNewParameters(serialized);
  const uint64_t L = c.db->getmaxFileBytesize();
  const uint64_t ct = server_crypto->getPublicParameters().getCiphertextBitsize() / 8;
  imported_database_t saved;
  saved.imported_database_ptr = NULL;
  bool ok[2] = {false, false};
  double reply_s[2] = {0, 0};
  size_t nrep[2] = {0, 0};
  for (int session = 0; session < 2; session++) {
    const uint64_t chosen = session == 0 ? c.chosen : c.chosen2;
    GenericPIRReplyGenerator *gen = PIRReplyGeneratorFactory::getPIRReplyGenerator("LWE", c.params, c.db);
    gen->setCryptoMethod(server_crypto);
    Session s{gen, server_crypto, &c.params, client.query(chosen), ct, gen->computeReplySizeInChunks(L), {}};
    pthread_t down, up;
    pthread_create(&down, nullptr, download, &s);
    pthread_create(&up, nullptr, upload, &s);
    const double t0 = now_s();
    if (session == 0)
      saved = gen->generateReplyGeneric(true);  // driven mode keeps the imported database
    else
      gen->generateReplyGenericFromData(saved);
    pthread_join(down, nullptr);
    pthread_join(up, nullptr);
    reply_s[session] = now_s() - t0;
    nrep[session] = s.replies.size();
    write_file(dir + (session == 0 ? "/replies.bin" : "/replies2.bin"), concat(s.replies, ct));
    ok[session] = client.extract(c.db, s.replies, chosen);
    delete gen;
  }
  dprintf(g_result_fd, "{\"mode\": \"server\", \"replies\": %zu, \"replies2\": %zu, \"kept_database\": %d, \"reply_s\": %.4f, "
         "\"reply2_s\": %.4f, \"extract_ok\": %d, \"extract2_ok\": %d}\n",
         nrep[0], nrep[1], saved.imported_database_ptr != NULL ? 1 : 0, reply_s[0], reply_s[1], ok[0] ? 1 : 0,
         ok[1] ? 1 : 0);
  delete server_crypto;
  return ok[0] && ok[1] ? 0 : 1;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: xpir_simplepir libpir|server <case 1-9> <dir>\n");
    return 2;
  }
  const std::string mode = argv[1], dir = argv[3];
  const int k = atoi(argv[2]);
  // DBDirectoryProcessor reads "db/" relative to the working directory.
  if (chdir(dir.c_str()) != 0) {
    fprintf(stderr, "xpir_simplepir: cannot enter %s\n", dir.c_str());
    return 2;
  }
  // XPIR prints progress on stdout: send it to stderr and keep the real stdout for the
  // one JSON result line.
  fflush(stdout);
  g_result_fd = dup(1);
  dup2(2, 1);
  xpir_ref_set_seed(4242 + (uint64_t)k);
  Case c = make_case(k, ".");
  return mode == "server" ? run_server(c, ".") : run_libpir(c, ".");
}
