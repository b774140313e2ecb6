// Host-side parameter set and NTT tables (the role of NFLlib::configureNTT,
// crypto/NFLlib.cpp:44-194), built once per (N, m) context and uploaded to HBM.
#include "params.h"

#include <math.h>

namespace xpir {

const uint64_t kModuli[kMaxModuli] = {
    2305843009213317121ULL, 2305843009213120513ULL, 2305843009212694529ULL, 2305843009212399617ULL,
    2305843009211662337ULL, 2305843009211596801ULL, 2305843009211400193ULL, 2305843009210580993ULL,
    2305843009210515457ULL, 2305843009210023937ULL, 2305843009209057281ULL, 2305843009208795137ULL,
    2305843009208713217ULL, 2305843009208123393ULL, 2305843009207468033ULL, 2305843009206976513ULL,
    2305843009206845441ULL};
const uint64_t kRoots2p14[kMaxModuli] = {
    1187132827279672845ULL, 753478288701480417ULL,  717492273700781398ULL,  1965831349000139179ULL,
    2188074825493578002ULL, 232964966911499637ULL,  395215708149128273ULL,  241993652537061162ULL,
    370764889455808762ULL,  1598724739621481826ULL, 610870591815427803ULL,  1880981984715338041ULL,
    1389374064030612248ULL, 1508488901479281364ULL, 2111887543055470169ULL, 2020509703903079203ULL,
    1120240637471598814ULL};
const uint64_t kInv8192[kMaxModuli] = {
    2305561534236606511ULL, 2305561534236409927ULL, 2305561534235983995ULL, 2305561534235689119ULL,
    2305561534234951929ULL, 2305561534234886401ULL, 2305561534234689817ULL, 2305561534233870717ULL,
    2305561534233805189ULL, 2305561534233313729ULL, 2305561534232347191ULL, 2305561534232085079ULL,
    2305561534232003169ULL, 2305561534231413417ULL, 2305561534230758137ULL, 2305561534230266677ULL,
    2305561534230135621ULL};

namespace {

typedef unsigned __int128 u128;

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)(((u128)a * b) % p); }
uint64_t shoup_of(uint64_t y, uint64_t p) { return (uint64_t)(((u128)y << 64) / p); }

uint32_t ilog2(uint64_t x) {
  uint32_t r = 0;
  while (x > 1) {
    x >>= 1;
    r++;
  }
  return r;
}

// Powers of w for each butterfly layer of the lazy DIF NTT: N/2 powers of w, then N/4
// powers of w^2, ..., one power of w^(N/2): N-1 words, the N-th left zero.
void layer_powers(uint64_t *tab, uint64_t *tab_shoup, uint64_t w, uint32_t N, uint64_t p) {
  uint32_t o = 0;
  for (uint32_t K = N; K >= 2; K >>= 1) {
    uint64_t wi = 1;
    for (uint32_t i = 0; i < K / 2; i++, o++) {
      tab[o] = wi;
      tab_shoup[o] = shoup_of(wi, p);
      wi = mulmod(wi, w, p);
    }
    w = mulmod(w, w, p);
  }
  tab[N - 1] = 0;
  tab_shoup[N - 1] = 0;
}

}  // namespace

bool valid_shape(uint32_t N, uint32_t m) {
  return m >= 1 && m <= kMaxModuli && N >= kMinPolyDegree && N <= kMaxPolyDegree && (N & (N - 1)) == 0;
}

int32_t bits_per_coeff(uint32_t N, uint32_t m, uint32_t security_bits, uint64_t n0) {
  const double berr = (double)(uint64_t)(5ull * security_bits / 2);
  const double bits = floor(((double)(kModulusBits * m) - 1 - log2((double)n0) - log2(berr) - log2((double)N)) / 2.0);
  if (!(bits > 0)) return 0;
  return (int32_t)bits;
}

uint64_t polys_for_bits(uint64_t total_bits, uint32_t b, uint32_t N) {
  if (b == 0) return 0;
  return (uint64_t)ceil((double)total_bits / (double)((uint64_t)b * N));
}

uint64_t reply_count(uint64_t element_bytes, uint32_t alpha, uint32_t d, uint32_t b, uint32_t N, uint32_t m) {
  if (b == 0) return 0;
  unsigned int out = (unsigned int)ceil((double)element_bytes * 8 * alpha / (double)((uint64_t)b * N));
  const double ct_bytes = (double)ciphertext_bytes(N, m);
  const double abs_bytes = (double)((uint64_t)b * N / 8);
  for (uint32_t i = 1; i < d; i++) out = (unsigned int)ceil(out * ct_bytes / abs_bytes);
  return out;
}

bool build_params(uint32_t N, uint32_t m, uint32_t b, ParamSet *ps, std::vector<uint64_t> *tables) {
  if (!valid_shape(N, m) || b == 0 || b > 4 * 56) return false;
  ps->N = N;
  ps->log_n = ilog2(N);
  ps->m = m;
  ps->b = b;
  tables->assign((size_t)m * kTableSlots * N, 0);
  for (uint32_t c = 0; c < m; c++) {
    const uint64_t p = kModuli[c];
    if (!shoup_factor_ok(p)) return false;
    ModulusConsts &mc = ps->mod[c];
    const ShoupConst sc = make_shoup_const(p);
    mc.p = p;
    mc.shoup_k = sc.k;
    mc.shoup_delta = sc.delta;
    uint64_t t = 1;
    for (int i = 0; i < 4; i++) {
      mc.crt[i] = t;
      mc.crt_shoup[i] = shoup_of(t, p);
      t = mulmod(t, 1ull << 56, p);
    }
    uint64_t *blk = tables->data() + (size_t)c * kTableSlots * N;
    uint64_t *phi = blk + kPhi * N, *phi_s = blk + kPhiShoup * N;
    uint64_t *iphi = blk + kInvPhi * N, *iphi_s = blk + kInvPhiShoup * N;
    // phi is a primitive 2N-th root: the 2^14-th root squared 13 - log2 N times.
    uint64_t root = kRoots2p14[c];
    for (int i = 0; i < 13 - (int)ps->log_n; i++) root = mulmod(root, root, p);
    t = 1;
    for (uint32_t i = 0; i < N; i++) {
      phi[i] = t;
      phi_s[i] = shoup_of(t, p);
      t = mulmod(t, root, p);
    }
    const uint64_t inv_root = mulmod(t, phi[N - 1], p);  // phi^N * phi^(N-1) = phi^-1
    t = mulmod(kInv8192[c], kMaxPolyDegree / N, p);       // N^-1
    for (uint32_t i = 0; i < N; i++) {
      iphi[i] = t;
      iphi_s[i] = shoup_of(t, p);
      t = mulmod(t, inv_root, p);
    }
    layer_powers(blk + kOmega * N, blk + kOmegaShoup * N, mulmod(root, root, p), N, p);
    layer_powers(blk + kInvOmega * N, blk + kInvOmegaShoup * N, mulmod(inv_root, inv_root, p), N, p);
  }
  return true;
}

}  // namespace xpir
