// Modular arithmetic of the NFLLWE path, shared by host and device code.
//
// Every function reproduces the exact bit pattern of the reference's lazy arithmetic
// (values are NOT canonical residues; see crypto/NFLlib.hpp:238-321).  Nothing here may
// "clean up" a value with a % p: the reply accumulators and NTT outputs are compared
// bit for bit with XPIR's CPU results.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define XPIR_HD __host__ __device__ __forceinline__
#else
#define XPIR_HD inline
#endif

namespace xpir {

constexpr uint32_t kMaxModuli = 17;
constexpr uint32_t kMinPolyDegree = 512;   // crypto/NFLParams.cpp:43
constexpr uint32_t kMaxPolyDegree = 8192;  // crypto/NFLParams.cpp:44
constexpr uint32_t kModulusBits = 60;      // crypto/NFLParams.cpp:31

// High 64 bits of a 64x64-bit product.  On the device: the schoolbook product of 32-bit
// halves with explicit carry chains (mad.lo/madc.hi), one instruction per product fewer
// on B200 than the generic 64-bit high multiply (measured with ncu instruction counts;
// identical results).
XPIR_HD uint64_t mulhi(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  uint64_t r;
  asm("{\n .reg .u32 a0, a1, b0, b1, t0, t1, t2;\n"
      " mov.b64 {a0, a1}, %1;\n"
      " mov.b64 {b0, b1}, %2;\n"
      " mul.hi.u32 t0, a0, b0;\n"         // carry-in from the low product
      " mad.lo.cc.u32 t0, a0, b1, t0;\n"
      " madc.hi.u32 t1, a0, b1, 0;\n"
      " mad.lo.cc.u32 t0, a1, b0, t0;\n"
      " madc.hi.cc.u32 t1, a1, b0, t1;\n"
      " addc.u32 t2, 0, 0;\n"
      " mad.lo.cc.u32 t1, a1, b1, t1;\n"
      " madc.hi.u32 t2, a1, b1, t2;\n"
      " mov.b64 %0, {t1, t2};\n"
      "}\n"
      : "=l"(r)
      : "l"(a), "l"(b));
  return r;
#else
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// Shoup product without the final correction, given np = 2^64 - p:
// x*y - floor(x*ys/2^64)*p = x*y + q*np (mod 2^64), so that the second product
// accumulates onto the first in multiply-add instructions.  For ys = floor(y*2^64/p) and
// y < p the result lies in [0, 2p) for any 64-bit x.  Device code passes np through
// opaque() so that the compiler keeps this form instead of rewriting it back into a
// product and a subtraction.
//
// On the device the whole expression is one block of 32-bit multiply-adds (the high
// product's carry chain, then the low 64 bits of x*y + q*np): 16 issued instructions on
// B200 against 18.7 for the C++ form over mulhi (ncu instruction counts of the isolated
// primitive), bit-identical on 2^24 random and edge-case triples.
XPIR_HD uint64_t shoup_lazy_np(uint64_t x, uint64_t y, uint64_t ys, uint64_t np) {
#if defined(__CUDA_ARCH__)
  uint64_t r;
  asm("{\n .reg .u32 x0, x1, y0, y1, s0, s1, n0, n1, t0, q0, q1, l, h;\n"
      " mov.b64 {x0, x1}, %1;\n"
      " mov.b64 {y0, y1}, %2;\n"
      " mov.b64 {s0, s1}, %3;\n"
      " mov.b64 {n0, n1}, %4;\n"
      " mul.hi.u32 t0, x0, s0;\n"          // q = hi(x * ys), as in mulhi
      " mad.lo.cc.u32 t0, x0, s1, t0;\n"
      " madc.hi.u32 q0, x0, s1, 0;\n"
      " mad.lo.cc.u32 t0, x1, s0, t0;\n"
      " madc.hi.cc.u32 q0, x1, s0, q0;\n"
      " addc.u32 q1, 0, 0;\n"
      " mad.lo.cc.u32 q0, x1, s1, q0;\n"
      " madc.hi.u32 q1, x1, s1, q1;\n"
      " mul.lo.u32 l, x0, y0;\n"           // low 64 bits of x*y + q*np
      " mul.hi.u32 h, x0, y0;\n"
      " mad.lo.cc.u32 l, q0, n0, l;\n"
      " madc.hi.u32 h, q0, n0, h;\n"
      " mad.lo.u32 h, x0, y1, h;\n"
      " mad.lo.u32 h, x1, y0, h;\n"
      " mad.lo.u32 h, q0, n1, h;\n"
      " mad.lo.u32 h, q1, n0, h;\n"
      " mov.b64 %0, {l, h};\n"
      "}\n"
      : "=l"(r)
      : "l"(x), "l"(y), "l"(ys), "l"(np));
  return r;
#else
  return x * y + mulhi(x, ys) * np;
#endif
}

// The same product given p (on the device through the multiply-add form above).
XPIR_HD uint64_t shoup_lazy(uint64_t x, uint64_t y, uint64_t ys, uint64_t p) {
#if defined(__CUDA_ARCH__)
  return shoup_lazy_np(x, y, ys, 0 - p);
#else
  return x * y - mulhi(x, ys) * p;
#endif
}

// A value the compiler cannot see through (a register move on the device).
XPIR_HD uint64_t opaque(uint64_t v) {
#if defined(__CUDA_ARCH__)
  asm volatile("mov.b64 %0, %0;" : "+l"(v));
#endif
  return v;
}

// mulmodShoup (crypto/NFLlib.hpp:282-289): the lazy product with one conditional
// subtraction.
XPIR_HD uint64_t shoup_mul(uint64_t x, uint64_t y, uint64_t ys, uint64_t p) {
  uint64_t r = shoup_lazy(x, y, ys, p);
  return r >= p ? r - p : r;
}

// mulandaddShoup (crypto/NFLlib.hpp:303-321): rop += x*y - q*p (mod 2^64), then at most
// one subtraction of p.
XPIR_HD uint64_t shoup_mac(uint64_t rop, uint64_t x, uint64_t y, uint64_t ys, uint64_t p) {
  rop += shoup_lazy(x, y, ys, p);
  return rop >= p ? rop - p : rop;
}

// Constants for computing the Shoup factor floor(y*2^64/p) of a query word without a
// 128-by-64-bit division.  Write 2^64 = k*p + delta (k = floor(2^64/p)).  Then
//   floor(y*2^64/p) = k*y + floor(y*delta/p).
// With z = y*delta (< 2^96 for delta < 2^32) and p <= 2^61, q0 = floor(z/2^61) is at
// most floor(z/p) and, when z*(2^61-p) < p*2^61, at least floor(z/p) - 1; the remainder
// z - q0*p lies in [0, 2p) and decides between the two.  shoup_factor_ok() checks these
// conditions for a modulus; all 17 XPIR moduli (p = 2^61 - i*2^14 + 1) satisfy them.
struct ShoupConst {
  uint64_t p;
  uint64_t k;      // floor(2^64 / p)
  uint64_t delta;  // 2^64 - k*p
};

inline bool shoup_factor_ok(uint64_t p) {
  if (p == 0 || p > (1ULL << 61) || p <= (1ULL << 59)) return false;
  unsigned __int128 two64 = (unsigned __int128)1 << 64;
  uint64_t k = (uint64_t)(two64 / p);
  unsigned __int128 delta = two64 - (unsigned __int128)k * p;
  if (delta >= ((unsigned __int128)1 << 32)) return false;
  // z < 2^64*delta, so z*(2^61-p) < p*2^61 holds for every z when
  // 2^64*delta*(2^61-p) <= p*2^61, i.e. 8*delta*(2^61-p) <= p.
  unsigned __int128 lhs = (unsigned __int128)8 * delta * ((1ULL << 61) - p);
  return lhs <= (unsigned __int128)p;
}

inline ShoupConst make_shoup_const(uint64_t p) {
  unsigned __int128 two64 = (unsigned __int128)1 << 64;
  ShoupConst s;
  s.p = p;
  s.k = (uint64_t)(two64 / p);
  s.delta = (uint64_t)(two64 - (unsigned __int128)s.k * p);
  return s;
}

// floor(y * 2^64 / p) mod 2^64, exact for every 64-bit y (the reference truncates the
// 128-bit quotient to 64 bits the same way, PIRReplyGeneratorNFL_internal.cpp:764).
XPIR_HD uint64_t shoup_factor(uint64_t y, uint64_t p, uint64_t k, uint64_t delta) {
  const uint64_t zlo = y * delta;
  const uint64_t zhi = mulhi(y, delta);
  const uint64_t q0 = (zhi << 3) | (zlo >> 61);
  const uint64_t rem = zlo - q0 * p;
  return k * y + q0 + (rem >= p ? 1 : 0);
}

// The same factor for moduli with k = 8 and delta < 2^26 (all 17 XPIR moduli), from
// 32x32-bit partial products only.  With y = yh*2^32 + yl:
//   A = yl*delta < 2^58,  B = yh*delta < 2^58,  z = y*delta = B*2^32 + A < 2^90,
//   q0 = floor(z / 2^61) = floor((B + floor(A/2^32)) / 2^29) < 2^30,
// and z mod 2^64 = A + B*2^32 (mod 2^64).  The remainder z - q0*p is in [0, 2p) (see
// shoup_factor_ok), so floor(z/p) = q0 + [z - q0*p >= p].
inline bool shoup_factor8_ok(uint64_t p) {
  if (!shoup_factor_ok(p)) return false;
  const ShoupConst s = make_shoup_const(p);
  return s.k == 8 && s.delta < (1ull << 26);
}

XPIR_HD uint64_t shoup_factor8(uint64_t y, uint64_t p, uint32_t delta) {
  const uint64_t A = (uint64_t)(uint32_t)y * delta;
  const uint64_t B = (uint64_t)(uint32_t)(y >> 32) * delta;
  const uint32_t q0 = (uint32_t)((B + (A >> 32)) >> 29);
  const uint64_t zlo = A + (B << 32);
  const uint64_t rem = zlo - (uint64_t)q0 * p;
  return (y << 3) + q0 + (rem >= p ? 1u : 0u);
}

// shoup_factor8 with np = 2^64 - p supplied (see shoup_lazy_np).  The correction
// [z - q0*p >= p] is read from the sign of r = z - (q0+1)*p = z + (q0+1)*np: since
// z - q0*p lies in [0, 2p) and 2p < 2^63, r is negative (top bit set) exactly when no
// correction is due.  Three instructions fewer than the compare on B200.
//
// On the device the same steps are spelled out on 32-bit halves, forming only the top
// word of r (its sign is all that is used): 13 issued instructions on B200 against 25 for
// the 64-bit C++ form (ncu instruction counts of the isolated primitive), bit-identical
// on 2^24 words x the 17 moduli.
XPIR_HD uint64_t shoup_factor8_np(uint64_t y, uint64_t p, uint64_t np, uint32_t delta) {
  (void)p;
#if defined(__CUDA_ARCH__)
  uint64_t r;
  asm("{\n .reg .u32 yl, yh, al, ah, bl, bh, sl, sh, q, rl, rh, nl, nh, sg, l, h;\n"
      " .reg .u64 A, B;\n"
      " mov.b64 {yl, yh}, %1;\n"
      " mov.b64 {nl, nh}, %2;\n"
      " mul.wide.u32 A, yl, %3;\n"           // A = yl * delta
      " mul.wide.u32 B, yh, %3;\n"           // B = yh * delta
      " mov.b64 {al, ah}, A;\n"
      " mov.b64 {bl, bh}, B;\n"
      " add.cc.u32 sl, bl, ah;\n"             // B + (A >> 32)
      " addc.u32 sh, bh, 0;\n"
      " shf.r.clamp.b32 q, sl, sh, 29;\n"     // q1 = (B + (A >> 32)) >> 29, + 1
      " add.u32 q, q, 1;\n"
      " mad.lo.cc.u32 rl, q, nl, al;\n"       // top word of A + (B << 32) + q1 * np
      " madc.hi.u32 rh, q, nl, ah;\n"
      " mad.lo.u32 rh, q, nh, rh;\n"
      " add.u32 rh, rh, bl;\n"
      " shr.u32 sg, rh, 31;\n"                // q1 - (r >> 63)
      " sub.u32 q, q, sg;\n"
      " shl.b32 l, yl, 3;\n"                  // (y << 3) + that
      " shf.l.clamp.b32 h, yl, yh, 3;\n"
      " add.cc.u32 l, l, q;\n"
      " addc.u32 h, h, 0;\n"
      " mov.b64 %0, {l, h};\n"
      "}\n"
      : "=l"(r)
      : "l"(y), "l"(np), "r"(delta));
  return r;
#else
  const uint64_t A = (uint64_t)(uint32_t)y * delta;
  const uint64_t B = (uint64_t)(uint32_t)(y >> 32) * delta;
  const uint32_t q1 = (uint32_t)((B + (A >> 32)) >> 29) + 1;
  const uint64_t r = A + (B << 32) + (uint64_t)q1 * np;
  return (y << 3) + (q1 - (uint32_t)(r >> 63));
#endif
}

}  // namespace xpir
