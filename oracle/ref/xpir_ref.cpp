// xpir_ref: command-line driver over the XPIR reference sources, compiled unchanged.
//
// Test infrastructure only (the parity checker).  Every computation below goes through
// the reference's own public libpir API and crypto classes, following the flow of
// apps/simplepir/simplePIR.cpp:3-182 (crypto setup -> PIRQueryGenerator ->
// PIRReplyGenerator importData/generateReply -> PIRReplyExtraction).  The driver only
// supplies inputs (a seeded DBVectorProcessor database, optional fixed queries) and
// writes the reference's outputs to files so the CUDA path can be compared bit for bit.
//
// Commands (all binary files are raw little-endian):
//   run      full PIR round trip; dumps query, imported DB, replies, recovered element
//   bench    one query, one import, then repeated timed replies (the benchmark's reference arm)
//   querygen the client's query generation alone, timed
//   extract  decrypt a given reply (e.g. one produced on the GPU) with the seeded key
//   key      write the seeded secret key (NTT domain) for the oracle's and GPU's decryption
//   tables   dump the NTT tables built by NFLlib::configureNTT (crypto/NFLlib.cpp:44-194)
//   bitsplit NFLlib::bitsplitter (+CRT) output, before the NTT (crypto/NFLlib.cpp:846-876)
//   deser    NFLlib::deserializeDataNFL output (bitsplit + CRT + nttAndPowPhi)
//   ntt      NFLlib::nttAndPowPhi on raw polynomials (crypto/NFLlib.hpp:597-608)
//   info     absorption/ciphertext sizes for a parameter set and n[0]
//
// White-box access to NFLlib's private tables and bitsplitter is obtained in this
// translation unit only, by compiling the reference headers with private/protected
// treated as public; the reference sources themselves are compiled unchanged.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <fstream>
#include <functional>
#include <iostream>
#include <iterator>
#include <limits>
#include <map>
#include <memory>
#include <random>
#include <set>
#include <sstream>
#include <string>
#include <tuple>
#include <utility>
#include <vector>
#include <fcntl.h>
#include <unistd.h>
#include <omp.h>
#include <gmp.h>
#include <boost/thread.hpp>
#include <boost/signals2.hpp>
#include <boost/algorithm/string.hpp>
#include <boost/pending/queue.hpp>
#include <boost/interprocess/sync/interprocess_semaphore.hpp>

#define private public
#define protected public
#include "libpir.hpp"
#undef private
#undef protected

extern "C" void xpir_ref_set_seed(uint64_t seed);

namespace {

int g_result_fd = 1;

// printf-style output of the JSON result line onto the saved real stdout.
template <class... T>
void result(const char *fmt, T... v) {
  dprintf(g_result_fd, fmt, v...);
}

struct Args {
  std::map<std::string, std::string> kv;
  bool has(const std::string &k) const { return kv.count(k) != 0; }
  std::string str(const std::string &k, const std::string &def = "") const {
    auto it = kv.find(k);
    return it == kv.end() ? def : it->second;
  }
  uint64_t u64(const std::string &k, uint64_t def = 0) const {
    auto it = kv.find(k);
    return it == kv.end() ? def : strtoull(it->second.c_str(), nullptr, 10);
  }
};

Args parse(int argc, char **argv) {
  Args a;
  for (int i = 2; i < argc; i++) {
    std::string k = argv[i];
    if (k.rfind("--", 0) != 0) continue;
    k = k.substr(2);
    if (i + 1 < argc && std::string(argv[i + 1]).rfind("--", 0) != 0) {
      a.kv[k] = argv[++i];
    } else {
      a.kv[k] = "1";
    }
  }
  return a;
}

std::vector<unsigned char> read_file(const std::string &path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    fprintf(stderr, "xpir_ref: cannot read %s\n", path.c_str());
    exit(2);
  }
  return std::vector<unsigned char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

void write_file(const std::string &path, const void *data, size_t n) {
  FILE *f = fopen(path.c_str(), "wb");
  if (!f || fwrite(data, 1, n, f) != n) {
    fprintf(stderr, "xpir_ref: cannot write %s\n", path.c_str());
    exit(2);
  }
  fclose(f);
}

// PIRParameters from --alpha --d --n n0,n1,... --params (pir/PIRParameters.hpp:24-29).
PIRParameters pir_params(const Args &a) {
  PIRParameters p;
  p.alpha = (unsigned)a.u64("alpha", 1);
  p.d = (unsigned)a.u64("d", 1);
  for (int i = 0; i < MAX_REC_LVL; i++) p.n[i] = 0;
  std::vector<std::string> f;
  boost::algorithm::split(f, a.str("n", "1"), boost::algorithm::is_any_of(","));
  for (size_t i = 0; i < f.size() && i < MAX_REC_LVL; i++) p.n[i] = (unsigned)strtoul(f[i].c_str(), nullptr, 10);
  p.crypto_params = a.str("params", "LWE:80:1024:60");
  return p;
}

// Crypto setup exactly as simplePIR.cpp:12-18: factory, then absorption sized for n[0].
HomomorphicCrypto *make_crypto(const Args &a, const PIRParameters &p) {
  xpir_ref_set_seed(a.u64("keyseed", 1));
  HomomorphicCrypto *crypto = HomomorphicCryptoFactory::getCryptoMethod(p.crypto_params);
  crypto->setandgetAbsBitPerCiphertext(p.n[0]);
  return crypto;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void print_info(NFLLWE *lwe, const PIRParameters &p) {
  AbstractPublicParameters &pp = lwe->getPublicParameters();
  result("{\"poly_degree\": %u, \"nb_moduli\": %u, \"abs_bits\": %u, \"bits_per_coeff\": %u, \"ct_bits\": %u",
         lwe->getpolyDegree(), (unsigned)lwe->getnbModuli(), pp.getAbsorptionBitsize(),
         pp.getAbsorptionBitsize() / lwe->getpolyDegree(), pp.getCiphertextBitsize());
  (void)p;
}

// Database: F elements of L bytes each, read from --db (DBVectorProcessor,
// pir/dbhandlers/DBVectorProcessor.cpp:34-110).
std::vector<element_t> *load_db(const Args &a) {
  uint64_t F = a.u64("nfiles"), L = a.u64("eltbytes");
  std::vector<unsigned char> raw = read_file(a.str("db"));
  if (raw.size() < F * L) {
    fprintf(stderr, "xpir_ref: db file too small\n");
    exit(2);
  }
  auto *elts = new std::vector<element_t>();
  elts->reserve(F);
  for (uint64_t i = 0; i < F; i++) elts->push_back(Element(std::to_string(i), L, (char *)raw.data() + i * L));
  return elts;
}

int cmd_run(const Args &a) {
  PIRParameters params = pir_params(a);
  HomomorphicCrypto *crypto = make_crypto(a, params);
  NFLLWE *lwe = dynamic_cast<NFLLWE *>(crypto);
  const uint64_t L = a.u64("eltbytes");
  const uint64_t chosen = a.u64("chosen", 0);
  const uint64_t ct_bytes = crypto->getPublicParameters().getCiphertextBitsize() / 8;
  uint64_t nq = 0;
  for (unsigned i = 0; i < params.d; i++) nq += params.n[i];

  std::vector<element_t> *elts = load_db(a);
  DBVectorProcessor db(*elts);

  // Query: the reference's PIRQueryGenerator (simplePIR.cpp:26-31), or a fixed query.
  std::vector<char *> query(nq, nullptr);
  double t0 = now_s();
  if (a.has("query-in")) {
    std::vector<unsigned char> q = read_file(a.str("query-in"));
    if (q.size() < nq * ct_bytes) {
      fprintf(stderr, "xpir_ref: query file too small\n");
      return 2;
    }
    for (uint64_t i = 0; i < nq; i++) {
      query[i] = (char *)malloc(ct_bytes);
      memcpy(query[i], q.data() + i * ct_bytes, ct_bytes);
    }
  } else {
    PIRQueryGenerator q_generator(params, *crypto);
    q_generator.generateQuery(chosen);
    for (uint64_t i = 0; i < nq; i++) q_generator.popQuery(&query[i]);
  }
  double t_query = now_s() - t0;
  if (a.has("query-out")) {
    std::vector<unsigned char> q(nq * ct_bytes);
    for (uint64_t i = 0; i < nq; i++) memcpy(q.data() + i * ct_bytes, query[i], ct_bytes);
    write_file(a.str("query-out"), q.data(), q.size());
  }

  // Reply generation (simplePIR.cpp:42-68): pushQuery takes ownership of each buffer.
  PIRReplyGenerator *r_generator = new PIRReplyGenerator(params, *crypto, &db);
  for (uint64_t i = 0; i < nq; i++) r_generator->pushQuery(query[i]);
  t0 = now_s();
  imported_database *imported_db = r_generator->importData(0, L);
  double t_import = now_s() - t0;

  const uint64_t N = lwe->getpolyDegree(), m = lwe->getnbModuli();
  if (a.has("imported-out")) {
    lwe_in_data *in = (lwe_in_data *)imported_db->imported_database_ptr;
    uint64_t P = imported_db->polysPerElement, E = imported_db->nbElements;
    std::vector<uint64_t> out(E * P * m * N);
    for (uint64_t e = 0; e < E; e++)
      for (uint64_t j = 0; j < P; j++) memcpy(&out[(e * P + j) * m * N], in[e].p[j], m * N * 8);
    write_file(a.str("imported-out"), out.data(), out.size() * 8);
  }

  t0 = now_s();
  r_generator->generateReply(imported_db);
  double t_reply = now_s() - t0;

  uint64_t nrep = r_generator->getnbRepliesGenerated();
  std::vector<char *> replies;
  char *rep;
  while (r_generator->popReply(&rep)) replies.push_back(rep);
  if (a.has("reply-out")) {
    std::vector<unsigned char> r(replies.size() * ct_bytes);
    for (size_t i = 0; i < replies.size(); i++) memcpy(r.data() + i * ct_bytes, replies[i], ct_bytes);
    write_file(a.str("reply-out"), r.data(), r.size());
  }

  // Extraction (simplePIR.cpp:121-166).
  int ok = -1;
  double t_extract = 0;
  if (!a.has("skip-extract")) {
    t0 = now_s();
    PIRReplyExtraction *r_extractor = new PIRReplyExtraction(params, *crypto);
    for (char *x : replies) r_extractor->pushEncryptedReply(x);
    replies.clear();
    r_extractor->extractReply(L);
    uint64_t pb = r_extractor->getPlaintextReplyBytesize();
    uint64_t np = r_extractor->getnbPlaintextReplies(L);
    char *plain = (char *)calloc(np * pb, 1), *outp = plain, *tmp;
    while (r_extractor->popPlaintextResult(&tmp)) {
      memcpy(outp, tmp, pb);
      outp += pb;
      free(tmp);
    }
    t_extract = now_s() - t0;
    char *db_element = (char *)calloc(L * params.alpha, 1);
    db.readAggregatedStream(chosen, params.alpha, 0, L, db_element);
    ok = memcmp(plain, db_element, L * params.alpha) == 0 ? 1 : 0;
    if (a.has("plain-out")) write_file(a.str("plain-out"), plain, L * params.alpha);
    free(db_element);
    free(plain);
    delete r_extractor;
  }
  for (char *x : replies) free(x);

  print_info(lwe, params);
  result(", \"polys_per_element\": %llu, \"nb_elements\": %llu, \"n_replies\": %llu, \"query_s\": %.6f, "
         "\"import_s\": %.6f, \"reply_s\": %.6f, \"extract_s\": %.6f, \"extract_ok\": %d, \"omp_threads\": %d}\n",
         (unsigned long long)imported_db->polysPerElement, (unsigned long long)imported_db->nbElements,
         (unsigned long long)nrep, t_query, t_import, t_reply, t_extract, ok, omp_get_max_threads());
  delete imported_db;
  r_generator->freeQueries();
  delete r_generator;
  delete crypto;
  delete elts;
  return ok == 0 ? 1 : 0;
}

// Repeated replies against one imported database, the way a server answers successive
// queries: the reference's query (PIRQueryGenerator) is pushed once, the database is
// imported once, then generateReply runs --warmup + --reps times on the same generator,
// each timed with omp_get_wtime at the boundaries the reference prints
// (PIRReplyGeneratorNFL_internal.cpp:354-444).  The benchmark's reference arm.
int cmd_bench(const Args &a) {
  PIRParameters params = pir_params(a);
  HomomorphicCrypto *crypto = make_crypto(a, params);
  NFLLWE *lwe = dynamic_cast<NFLLWE *>(crypto);
  const uint64_t L = a.u64("eltbytes");
  const uint64_t reps = a.u64("reps", 1), warmup = a.u64("warmup", 0);
  std::vector<element_t> *elts = load_db(a);
  DBVectorProcessor db(*elts);
  double t0 = omp_get_wtime();
  PIRQueryGenerator q_generator(params, *crypto);
  q_generator.generateQuery(a.u64("chosen", 0));
  const double t_query = omp_get_wtime() - t0;
  PIRReplyGenerator *r_generator = new PIRReplyGenerator(params, *crypto, &db);
  char *q;
  t0 = omp_get_wtime();
  while (q_generator.popQuery(&q)) r_generator->pushQuery(q);
  const double t_push = omp_get_wtime() - t0;
  t0 = omp_get_wtime();
  imported_database *imported_db = r_generator->importData(0, L);
  const double t_import = omp_get_wtime() - t0;
  std::vector<double> reply_s;
  uint64_t nrep = 0;
  for (uint64_t i = 0; i < warmup + reps; i++) {
    t0 = omp_get_wtime();
    r_generator->generateReply(imported_db);
    const double t = omp_get_wtime() - t0;
    if (i >= warmup) reply_s.push_back(t);
    char *rep;
    nrep = 0;
    while (r_generator->popReply(&rep)) {
      free(rep);
      nrep++;
    }
  }
  print_info(lwe, params);
  result(", \"polys_per_element\": %llu, \"nb_elements\": %llu, \"n_replies\": %llu, \"query_s\": %.6f, "
         "\"push_s\": %.6f, \"import_s\": %.6f, \"omp_threads\": %d, \"reply_s\": [",
         (unsigned long long)imported_db->polysPerElement, (unsigned long long)imported_db->nbElements,
         (unsigned long long)nrep, t_query, t_push, t_import, omp_get_max_threads());
  for (size_t i = 0; i < reply_s.size(); i++) result(i ? ", %.6f" : "%.6f", reply_s[i]);
  result("]}\n");
  delete imported_db;
  r_generator->freeQueries();
  delete r_generator;
  delete crypto;
  delete elts;
  return 0;
}

// Client-side query generation alone (PIRQueryGenerator::generateQuery, pir/libpir.cpp:45-60),
// timed with omp_get_wtime: the reference side of the benchmark's query-generation workload.
int cmd_querygen(const Args &a) {
  PIRParameters params = pir_params(a);
  HomomorphicCrypto *crypto = make_crypto(a, params);
  double t0 = omp_get_wtime();
  PIRQueryGenerator q_generator(params, *crypto);
  q_generator.generateQuery(a.u64("chosen", 0));
  const double t_query = omp_get_wtime() - t0;
  uint64_t count = 0;
  char *q;
  while (q_generator.popQuery(&q)) {
    free(q);
    count++;
  }
  print_info(dynamic_cast<NFLLWE *>(crypto), params);
  result(", \"ciphertexts\": %llu, \"query_s\": %.6f, \"omp_threads\": %d}\n", (unsigned long long)count, t_query,
         omp_get_max_threads());
  delete crypto;
  return 0;
}

// Decrypt given replies with the seeded key (PIRReplyExtraction, libpir.cpp:171-201).
int cmd_extract(const Args &a) {
  PIRParameters params = pir_params(a);
  HomomorphicCrypto *crypto = make_crypto(a, params);
  const uint64_t L = a.u64("eltbytes");
  const uint64_t ct_bytes = crypto->getPublicParameters().getCiphertextBitsize() / 8;
  std::vector<unsigned char> r = read_file(a.str("reply-in"));
  uint64_t nrep = r.size() / ct_bytes;
  PIRReplyExtraction *r_extractor = new PIRReplyExtraction(params, *crypto);
  for (uint64_t i = 0; i < nrep; i++) {
    char *x = (char *)malloc(ct_bytes);
    memcpy(x, r.data() + i * ct_bytes, ct_bytes);
    r_extractor->pushEncryptedReply(x);
  }
  const double t0 = omp_get_wtime();
  r_extractor->extractReply(L);
  const double t_extract = omp_get_wtime() - t0;
  uint64_t pb = r_extractor->getPlaintextReplyBytesize();
  uint64_t np = r_extractor->getnbPlaintextReplies(L);
  std::vector<char> plain(np * pb);
  char *outp = plain.data(), *tmp;
  while (r_extractor->popPlaintextResult(&tmp)) {
    memcpy(outp, tmp, pb);
    outp += pb;
    free(tmp);
  }
  write_file(a.str("plain-out"), plain.data(), L * params.alpha);
  delete r_extractor;
  delete crypto;
  result("{\"replies\": %llu, \"extract_s\": %.6f, \"omp_threads\": %d}\n", (unsigned long long)nrep, t_extract,
         omp_get_max_threads());
  return 0;
}

// The seeded secret key (NFLLWE::secretKey, crypto/NFLLWE.cpp:98-120): m*N words, NTT
// domain, written to --key-out.
int cmd_key(const Args &a) {
  PIRParameters params = pir_params(a);
  HomomorphicCrypto *crypto = make_crypto(a, params);
  NFLLWE *lwe = dynamic_cast<NFLLWE *>(crypto);
  const uint64_t words = (uint64_t)lwe->getnbModuli() * lwe->getpolyDegree();
  write_file(a.str("key-out"), lwe->getsecretKey()[0], words * 8);
  delete crypto;
  return 0;
}

int cmd_info(const Args &a) {
  PIRParameters params = pir_params(a);
  HomomorphicCrypto *crypto = make_crypto(a, params);
  print_info(dynamic_cast<NFLLWE *>(crypto), params);
  result("}\n");
  delete crypto;
  return 0;
}

// NTT tables of NFLlib::configureNTT, per modulus: modulus, then phis[N], shoupphis[N],
// omegas[N], shoupomegas[N], invpoly_times_invphis[N], shoupinvpoly_times_invphis[N],
// invomegas[N], shoupinvomegas[N], then inv_indexes[N] once.
int cmd_tables(const Args &a) {
  PIRParameters params = pir_params(a);
  HomomorphicCrypto *crypto = make_crypto(a, params);
  NFLlib &nfl = dynamic_cast<NFLLWE *>(crypto)->getnflInstance();
  const uint64_t N = nfl.getpolyDegree(), m = nfl.getnbModuli();
  std::vector<uint64_t> out;
  for (uint64_t c = 0; c < m; c++) {
    out.push_back(nfl.moduli[c]);
    out.insert(out.end(), nfl.phis[c], nfl.phis[c] + N);
    out.insert(out.end(), nfl.shoupphis[c], nfl.shoupphis[c] + N);
    out.insert(out.end(), nfl.omegas[c], nfl.omegas[c] + N);
    out.insert(out.end(), nfl.shoupomegas[c], nfl.shoupomegas[c] + N);
    out.insert(out.end(), nfl.invpoly_times_invphis[c], nfl.invpoly_times_invphis[c] + N);
    out.insert(out.end(), nfl.shoupinvpoly_times_invphis[c], nfl.shoupinvpoly_times_invphis[c] + N);
    out.insert(out.end(), nfl.invomegas[c], nfl.invomegas[c] + N);
    out.insert(out.end(), nfl.shoupinvomegas[c], nfl.shoupinvomegas[c] + N);
  }
  out.insert(out.end(), nfl.inv_indexes, nfl.inv_indexes + N);
  write_file(a.str("out"), out.data(), out.size() * 8);
  delete crypto;
  return 0;
}

// Buffers for the bit splitter: --nbufs k buffers of --bufbits bits each, stored back
// to back in --in, each padded to --bufstride bytes (default: ceil(bits/8)).
struct Buffers {
  std::vector<unsigned char> raw;
  std::vector<unsigned char *> ptrs;
};

Buffers load_buffers(const Args &a) {
  Buffers b;
  uint64_t k = a.u64("nbufs", 1), bits = a.u64("bufbits");
  uint64_t stride = a.u64("bufstride", (bits + 7) / 8);
  std::vector<unsigned char> in = read_file(a.str("in"));
  // Over-allocate: the reference reads whole 64-bit words past the last useful byte.
  b.raw.assign(k * stride + 64, 0);
  memcpy(b.raw.data(), in.data(), std::min<size_t>(in.size(), k * stride));
  for (uint64_t i = 0; i < k; i++) b.ptrs.push_back(b.raw.data() + i * stride);
  return b;
}

int cmd_bitsplit(const Args &a, bool ntt) {
  PIRParameters params = pir_params(a);
  HomomorphicCrypto *crypto = make_crypto(a, params);
  NFLLWE *lwe = dynamic_cast<NFLLWE *>(crypto);
  NFLlib &nfl = lwe->getnflInstance();
  const uint64_t N = nfl.getpolyDegree(), m = nfl.getnbModuli();
  unsigned b = lwe->getPublicParameters().getAbsorptionBitsize() / N;
  if (a.has("bits")) b = (unsigned)a.u64("bits");
  Buffers bufs = load_buffers(a);
  uint64_t k = a.u64("nbufs", 1), bits = a.u64("bufbits");
  uint64_t P = 0;
  poly64 *polys = nfl.deserializeDataNFL(bufs.ptrs.data(), k, bits, b, P);
  if (!ntt) {
    // Re-run only the splitter (deserializeDataNFL = bitsplitter + per-poly NTT).
    free(polys[0]);
    free(polys);
    uint64_t *split = nfl.bitsplitter(bufs.ptrs.data(), k, bits, b);
    write_file(a.str("out"), split, P * m * N * 8);
    free(split);
  } else {
    write_file(a.str("out"), polys[0], P * m * N * 8);
    free(polys[0]);
    free(polys);
  }
  result("{\"bits_per_coeff\": %u, \"polys\": %llu}\n", b, (unsigned long long)P);
  delete crypto;
  return 0;
}

int cmd_ntt(const Args &a) {
  PIRParameters params = pir_params(a);
  HomomorphicCrypto *crypto = make_crypto(a, params);
  NFLlib &nfl = dynamic_cast<NFLLWE *>(crypto)->getnflInstance();
  const uint64_t N = nfl.getpolyDegree(), m = nfl.getnbModuli();
  std::vector<unsigned char> in = read_file(a.str("in"));
  uint64_t np = in.size() / (m * N * 8);
  std::vector<uint64_t> x(np * m * N);
  memcpy(x.data(), in.data(), x.size() * 8);
  for (uint64_t i = 0; i < np; i++) nfl.nttAndPowPhi(&x[i * m * N]);
  write_file(a.str("out"), x.data(), x.size() * 8);
  delete crypto;
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: xpir_ref run|bench|querygen|extract|key|tables|bitsplit|deser|ntt|info [--key value ...]\n");
    return 2;
  }
  std::string cmd = argv[1];
  Args a = parse(argc, argv);
  // The reference prints progress with both printf and std::cout; send all of it to
  // stderr (or nowhere) and keep the real stdout for the one JSON result line.
  fflush(stdout);
  g_result_fd = dup(1);
  int sink = a.has("verbose") ? dup(2) : open("/dev/null", O_WRONLY);
  dup2(sink, 1);
  close(sink);
  if (cmd == "run") return cmd_run(a);
  if (cmd == "bench") return cmd_bench(a);
  if (cmd == "querygen") return cmd_querygen(a);
  if (cmd == "extract") return cmd_extract(a);
  if (cmd == "tables") return cmd_tables(a);
  if (cmd == "bitsplit") return cmd_bitsplit(a, false);
  if (cmd == "deser") return cmd_bitsplit(a, true);
  if (cmd == "ntt") return cmd_ntt(a);
  if (cmd == "info") return cmd_info(a);
  if (cmd == "key") return cmd_key(a);
  fprintf(stderr, "xpir_ref: unknown command %s\n", cmd.c_str());
  return 2;
}
