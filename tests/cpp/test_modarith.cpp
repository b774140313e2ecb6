// Host-side check of the engine's modular arithmetic (xpir_b200/csrc/modarith.cuh),
// compiled with g++: the division-free Shoup factor must equal floor(y*2^64/p) mod 2^64
// (the reference's u128 division, PIRReplyGeneratorNFL_internal.cpp:764) for every y, and
// the accumulate forms (given 2^64 - p) must equal the plain ones.
#include <stdio.h>
#include <stdlib.h>

#include <random>

#include "../../xpir_b200/csrc/modarith.cuh"
#include "../../xpir_b200/csrc/params.h"

int main() {
  std::mt19937_64 rng(12345);
  long checked = 0;
  for (unsigned c = 0; c < xpir::kMaxModuli; c++) {
    const uint64_t p = xpir::kModuli[c];
    if (!xpir::shoup_factor_ok(p)) {
      printf("modulus %u rejected\n", c);
      return 1;
    }
    const xpir::ShoupConst s = xpir::make_shoup_const(p);
    const uint64_t edge[] = {0, 1, 2, p - 2, p - 1, p, p + 1, 2 * p - 1, 2 * p, 3 * p + 7, (1ULL << 61) - 1,
                             1ULL << 61, (1ULL << 62) + 3, 1ULL << 63, ~0ULL - 1, ~0ULL};
    if (!xpir::shoup_factor8_ok(p)) {
      printf("modulus %u has no k=8 fast path\n", c);
      return 1;
    }
    auto check = [&](uint64_t y) {
      const uint64_t want = (uint64_t)(((unsigned __int128)y << 64) / p);
      const uint64_t got = xpir::shoup_factor(y, p, s.k, s.delta);
      const uint64_t got8 = xpir::shoup_factor8(y, p, (uint32_t)s.delta);
      const uint64_t got8n = xpir::shoup_factor8_np(y, p, 0 - p, (uint32_t)s.delta);
      // The accumulate form of the lazy product equals the subtract form for any x.
      const uint64_t x = rng();
      const uint64_t lazy = xpir::shoup_lazy(x, y, want, p);
      const uint64_t lazy_np = xpir::shoup_lazy_np(x, y, want, 0 - p);
      checked++;
      if (want != got || want != got8 || want != got8n || lazy != lazy_np) {
        printf("mismatch p=%llu y=%llu want=%llu got=%llu\n", (unsigned long long)p, (unsigned long long)y,
               (unsigned long long)want, (unsigned long long)got);
        exit(1);
      }
    };
    for (uint64_t y : edge) check(y);
    for (int i = 0; i < 200000; i++) check(rng() % p);
    for (int i = 0; i < 200000; i++) check(rng());
    // values right below and above multiples of p / 2^k boundaries
    for (int i = 0; i < 2000; i++) {
      uint64_t k = rng() % 8;
      check(k * p + (rng() % 3));
      check(k * p - 1 - (rng() % 3));
    }
  }
  printf("ok %ld\n", checked);
  return 0;
}
