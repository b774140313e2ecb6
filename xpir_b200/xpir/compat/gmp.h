/* Declarations of the public GMP 6 mpz API used by the XPIR reference sources.
 *
 * This header lets XPIR's own sources -- compiled unchanged, both as the parity checker
 * and with the B200 reply generator plugged in -- link against the GMP runtime library
 * that this image ships as libgmp.so.10 without development headers.  A normal XPIR
 * build uses the system's gmp.h instead.  Only documented public
 * types and functions are declared, under their exported __gmp names. */
#ifndef XPIR_REF_SHIM_GMP_H
#define XPIR_REF_SHIM_GMP_H

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned long mp_limb_t;
typedef long mp_size_t;
typedef unsigned long mp_bitcnt_t;

typedef struct {
  int _mp_alloc;
  int _mp_size;
  mp_limb_t *_mp_d;
} __mpz_struct;

typedef __mpz_struct mpz_t[1];
typedef __mpz_struct *mpz_ptr;
typedef const __mpz_struct *mpz_srcptr;

typedef enum { GMP_RAND_ALG_DEFAULT = 0, GMP_RAND_ALG_LC = GMP_RAND_ALG_DEFAULT } gmp_randalg_t;
typedef struct {
  mpz_t _mp_seed;
  gmp_randalg_t _mp_alg;
  union { void *_mp_lc; } _mp_algdata;
} __gmp_randstate_struct;
typedef __gmp_randstate_struct gmp_randstate_t[1];

#define mpz_init __gmpz_init
#define mpz_inits __gmpz_inits
#define mpz_init2 __gmpz_init2
#define mpz_init_set __gmpz_init_set
#define mpz_init_set_ui __gmpz_init_set_ui
#define mpz_clear __gmpz_clear
#define mpz_clears __gmpz_clears
#define mpz_set __gmpz_set
#define mpz_set_ui __gmpz_set_ui
#define mpz_get_ui __gmpz_get_ui
#define mpz_import __gmpz_import
#define mpz_export __gmpz_export
#define mpz_add __gmpz_add
#define mpz_add_ui __gmpz_add_ui
#define mpz_sub __gmpz_sub
#define mpz_sub_ui __gmpz_sub_ui
#define mpz_mul __gmpz_mul
#define mpz_mul_ui __gmpz_mul_ui
#define mpz_mul_2exp __gmpz_mul_2exp
#define mpz_mod __gmpz_mod
#define mpz_div __gmpz_fdiv_q
#define mpz_fdiv_q __gmpz_fdiv_q
#define mpz_divexact __gmpz_divexact
#define mpz_and __gmpz_and
#define mpz_cmp __gmpz_cmp
#define mpz_invert __gmpz_invert
#define mpz_ui_pow_ui __gmpz_ui_pow_ui
#define mpz_pow_ui __gmpz_pow_ui
#define mpz_powm __gmpz_powm
#define mpz_lcm __gmpz_lcm
#define mpz_bin_ui __gmpz_bin_ui
#define mpz_nextprime __gmpz_nextprime
#define mpz_sizeinbase __gmpz_sizeinbase
#define mpz_urandomb __gmpz_urandomb
#define gmp_randinit_default __gmp_randinit_default
#define gmp_randseed __gmp_randseed
#define gmp_randseed_ui __gmp_randseed_ui
#define gmp_randclear __gmp_randclear
#define gmp_printf __gmp_printf

void __gmpz_init(mpz_ptr);
void __gmpz_inits(mpz_ptr, ...);
void __gmpz_init2(mpz_ptr, mp_bitcnt_t);
void __gmpz_init_set(mpz_ptr, mpz_srcptr);
void __gmpz_init_set_ui(mpz_ptr, unsigned long);
void __gmpz_clear(mpz_ptr);
void __gmpz_clears(mpz_ptr, ...);
void __gmpz_set(mpz_ptr, mpz_srcptr);
void __gmpz_set_ui(mpz_ptr, unsigned long);
unsigned long __gmpz_get_ui(mpz_srcptr);
void __gmpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void *);
void *__gmpz_export(void *, size_t *, int, size_t, int, size_t, mpz_srcptr);
void __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_sub_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_mod(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_fdiv_q(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_divexact(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_and(mpz_ptr, mpz_srcptr, mpz_srcptr);
int __gmpz_cmp(mpz_srcptr, mpz_srcptr);
int __gmpz_invert(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_ui_pow_ui(mpz_ptr, unsigned long, unsigned long);
void __gmpz_pow_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_powm(mpz_ptr, mpz_srcptr, mpz_srcptr, mpz_srcptr);
void __gmpz_lcm(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_bin_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_nextprime(mpz_ptr, mpz_srcptr);
size_t __gmpz_sizeinbase(mpz_srcptr, int);
void __gmpz_urandomb(mpz_ptr, __gmp_randstate_struct *, mp_bitcnt_t);
void __gmp_randinit_default(__gmp_randstate_struct *);
void __gmp_randseed(__gmp_randstate_struct *, mpz_srcptr);
void __gmp_randseed_ui(__gmp_randstate_struct *, unsigned long);
void __gmp_randclear(__gmp_randstate_struct *);
int __gmp_printf(const char *, ...);

#ifdef __cplusplus
}
#endif

#endif
