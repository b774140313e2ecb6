// Seeded replacement for the reference's crypto/prng/randombytes.cpp (which reads
// /dev/urandom).  Linked in its place when the reference is compiled as the parity
// checker, so that secret keys, noise and the uniform "a" polynomials are reproducible:
// the reference's fastrandombytes() keys its Salsa20 stream from the first call here.
// Test infrastructure only.
#include <cstdint>
#include <cstdlib>

static uint64_t g_state = 0x9e3779b97f4a7c15ULL;

extern "C" void xpir_ref_set_seed(uint64_t seed) { g_state = seed * 0x2545F4914F6CDD1DULL + 0x9e3779b97f4a7c15ULL; }

static uint64_t splitmix64_next() {
  uint64_t z = (g_state += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

void randombytes(unsigned char *x, unsigned long long xlen) {
  while (xlen > 0) {
    uint64_t v = splitmix64_next();
    for (int i = 0; i < 8 && xlen > 0; i++, xlen--) *x++ = (unsigned char)(v >> (8 * i));
  }
}
