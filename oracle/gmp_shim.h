/*
 * gmp_shim.h -- hand-written declarations of the public GMP 6.x mpz API.
 *
 * TEST INFRASTRUCTURE ONLY.  This header is part of the CPU oracle: it is
 * used by oracle/oracle.c and by the C++ drop-in compile test, never by the
 * CUDA product library.
 *
 * The image ships the GMP runtime (libgmp.so.10, GMP 6.3.0) but not gmp.h.
 * The declarations below follow GMP's documented, stable public ABI: every
 * mpz_xxx function is exported as __gmpz_xxx, and mpz_t is a one-element
 * array of {int alloc; int size; mp_limb_t *d;}.  Only the functions the
 * reference calls on its CPU path (gap_common.cpp:60-65, gpu_testing.cu:171,
 * miller_rabin.h:39-54, overflow.cpp:124-168) plus a few helpers are listed;
 * oracle/include/gmp.h exposes them under the name <gmp.h> so the reference's
 * own gap_common.cpp and overflow.cpp compile against them (oracle/Makefile,
 * target ref).
 */
#ifndef PG_ORACLE_GMP_SHIM_H
#define PG_ORACLE_GMP_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned long mp_limb_t;
typedef unsigned long mp_bitcnt_t;

typedef struct {
    int _mp_alloc;
    int _mp_size;
    mp_limb_t *_mp_d;
} __mpz_struct;

typedef __mpz_struct mpz_t[1];
typedef __mpz_struct *mpz_ptr;
typedef const __mpz_struct *mpz_srcptr;

void __gmpz_init(mpz_ptr);
void __gmpz_inits(mpz_ptr, ...);
void __gmpz_init_set(mpz_ptr, mpz_srcptr);
void __gmpz_clear(mpz_ptr);
void __gmpz_clears(mpz_ptr, ...);
void __gmpz_set(mpz_ptr, mpz_srcptr);
void __gmpz_set_ui(mpz_ptr, unsigned long);
int __gmpz_set_str(mpz_ptr, const char *, int);
char *__gmpz_get_str(char *, int, mpz_srcptr);
void __gmpz_primorial_ui(mpz_ptr, unsigned long);
unsigned long __gmpz_tdiv_q_ui(mpz_ptr, mpz_srcptr, unsigned long);
unsigned long __gmpz_fdiv_ui(mpz_srcptr, unsigned long);
void __gmpz_mul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_sub_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mod(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_tdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_nextprime(mpz_ptr, mpz_srcptr);
int __gmpz_prevprime(mpz_ptr, mpz_srcptr);
int __gmpz_probab_prime_p(mpz_srcptr, int);
void __gmpz_powm(mpz_ptr, mpz_srcptr, mpz_srcptr, mpz_srcptr);
void __gmpz_powm_ui(mpz_ptr, mpz_srcptr, unsigned long, mpz_srcptr);
void __gmpz_ui_pow_ui(mpz_ptr, unsigned long, unsigned long);
void *__gmpz_export(void *, size_t *, int, size_t, int, size_t, mpz_srcptr);
void __gmpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void *);
size_t __gmpz_sizeinbase(mpz_srcptr, int);
double __gmpz_get_d_2exp(long *, mpz_srcptr);
int __gmpz_cmp(mpz_srcptr, mpz_srcptr);
int __gmpz_cmp_ui(mpz_srcptr, unsigned long);
unsigned long __gmpz_get_ui(mpz_srcptr);
mp_bitcnt_t __gmpz_scan1(mpz_srcptr, mp_bitcnt_t);
int __gmpz_tstbit(mpz_srcptr, mp_bitcnt_t);

#define mpz_init __gmpz_init
#define mpz_inits __gmpz_inits
#define mpz_init_set __gmpz_init_set
#define mpz_clear __gmpz_clear
#define mpz_clears __gmpz_clears
#define mpz_set __gmpz_set
#define mpz_set_ui __gmpz_set_ui
#define mpz_set_str __gmpz_set_str
#define mpz_get_str __gmpz_get_str
#define mpz_primorial_ui __gmpz_primorial_ui
#define mpz_tdiv_q_ui __gmpz_tdiv_q_ui
#define mpz_fdiv_ui __gmpz_fdiv_ui
#define mpz_mul_ui __gmpz_mul_ui
#define mpz_mul __gmpz_mul
#define mpz_add_ui __gmpz_add_ui
#define mpz_sub_ui __gmpz_sub_ui
#define mpz_add __gmpz_add
#define mpz_sub __gmpz_sub
#define mpz_mod __gmpz_mod
#define mpz_mul_2exp __gmpz_mul_2exp
#define mpz_tdiv_q_2exp __gmpz_tdiv_q_2exp
#define mpz_nextprime __gmpz_nextprime
#define mpz_prevprime __gmpz_prevprime
#define mpz_probab_prime_p __gmpz_probab_prime_p
#define mpz_powm __gmpz_powm
#define mpz_powm_ui __gmpz_powm_ui
#define mpz_ui_pow_ui __gmpz_ui_pow_ui
#define mpz_export __gmpz_export
#define mpz_import __gmpz_import
#define mpz_sizeinbase __gmpz_sizeinbase
#define mpz_get_d_2exp __gmpz_get_d_2exp
#define mpz_cmp __gmpz_cmp
#define mpz_cmp_ui __gmpz_cmp_ui
#define mpz_get_ui __gmpz_get_ui
#define mpz_scan1 __gmpz_scan1
#define mpz_tstbit __gmpz_tstbit
#define mpz_odd_p(z) ((z)->_mp_size != 0 && ((z)->_mp_d[0] & 1))

#ifdef __cplusplus
}
#endif

#endif /* PG_ORACLE_GMP_SHIM_H */
