// NFLLWE parameter set and NTT tables for the B200 reply engine (host side).
#pragma once

#include <stdint.h>

#include <vector>

#include "modarith.cuh"

namespace xpir {

// The reference's 60-bit moduli p_i = 2^61 - i*2^14 + 1, primitive 2^14-th roots of
// unity and inverses of 8192 (crypto/NFLParams.cpp:30,36,40).  The values must be the
// reference's: every NTT-domain word of the database and of the queries depends on them.
extern const uint64_t kModuli[kMaxModuli];
extern const uint64_t kRoots2p14[kMaxModuli];
extern const uint64_t kInv8192[kMaxModuli];

// Per-modulus table block, N words each, in this order (word offsets are multiples of N):
enum TableSlot : uint32_t {
  kPhi = 0,        // phi^i                       (crypto/NFLlib.cpp:94-101)
  kPhiShoup,       // floor(phi^i 2^64 / p)
  kOmega,          // forward twiddles, layer by layer: N/2 powers of w, N/4 of w^2, ...
  kOmegaShoup,     //                               (crypto/NFLlib.hpp:571-586)
  kInvPhi,         // N^-1 phi^-i                 (crypto/NFLlib.cpp:109-121)
  kInvPhiShoup,
  kInvOmega,       // inverse twiddles, same layout as kOmega
  kInvOmegaShoup,
  kTableSlots
};

// Constants the kernels need per modulus, passed by value as a kernel argument.
struct ModulusConsts {
  uint64_t p;
  uint64_t shoup_k;      // floor(2^64/p)          (query Shoup factors, modarith.cuh)
  uint64_t shoup_delta;  // 2^64 - k*p
  uint64_t crt[4];       // 2^(56 t) mod p          (crypto/NFLlib.cpp:890-897)
  uint64_t crt_shoup[4];
};

struct ParamSet {
  uint32_t N = 0;        // polynomial degree
  uint32_t log_n = 0;
  uint32_t m = 0;        // number of 60-bit moduli
  uint32_t b = 0;        // bits absorbed per coefficient
  ModulusConsts mod[kMaxModuli];
};

// Returns false if (N, m) is outside what the reference supports.
bool valid_shape(uint32_t N, uint32_t m);

// floor(((60m - 1) - log2 n0 - log2(5k/2) - log2 N) / 2), the reference's double
// arithmetic (crypto/NFLLWE.cpp:656-668; noise bound crypto/NFLLWE.cpp:84).
int32_t bits_per_coeff(uint32_t N, uint32_t m, uint32_t security_bits, uint64_t n0);

// ceil(total_bits / (b N)) in double, as crypto/NFLlib.cpp:379.
uint64_t polys_for_bits(uint64_t total_bits, uint32_t b, uint32_t N);

// computeReplySizeInChunks (pir/replyGenerator/PIRReplyGeneratorNFL_internal.cpp:667-679).
uint64_t reply_count(uint64_t element_bytes, uint32_t alpha, uint32_t d, uint32_t b, uint32_t N, uint32_t m);

// Bytes of one ciphertext [a][b] of m polys of N 64-bit words
// (NFLLWEPublicParameters.cpp:82-86,148-151).
inline uint64_t ciphertext_bytes(uint32_t N, uint32_t m) { return 2ull * 8ull * m * N; }

// Builds ParamSet constants and the host copy of the NTT tables (m * kTableSlots * N
// words), the equivalent of NFLlib::configureNTT (crypto/NFLlib.cpp:44-194).
bool build_params(uint32_t N, uint32_t m, uint32_t b, ParamSet *ps, std::vector<uint64_t> *tables);

}  // namespace xpir
