/* Declaration header for the subset of GMP's public, documented mpz API that the oracle and the
 * reference's own sources use. TEST INFRASTRUCTURE ONLY: it lets the oracle (and the reference's
 * lucaslehmer.cpp, compiled unchanged from its own source tree) link against the system's GMP
 * runtime (libgmp.so.10, GMP 6.3.0) on a machine that ships the library but not its development
 * header. Nothing in the product includes this file.
 *
 * Only names, the documented struct layouts of mpz_t / gmp_randstate_t and function signatures
 * are declared here; every function body lives in the GMP library itself. GMP's public macros map
 * mpz_foo to the exported symbol __gmpz_foo; the same mapping is written out below. */
#ifndef ORACLE_SHIM_GMP_H
#define ORACLE_SHIM_GMP_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned long mp_limb_t;
typedef unsigned long mp_bitcnt_t;
typedef long mp_size_t;

typedef struct {
    int _mp_alloc;
    int _mp_size;
    mp_limb_t* _mp_d;
} __mpz_struct;
typedef __mpz_struct mpz_t[1];
typedef __mpz_struct* mpz_ptr;
typedef const __mpz_struct* mpz_srcptr;

typedef struct {
    mpz_t _mp_seed;
    int _mp_alg;
    union {
        void* _mp_lc;
    } _mp_algdata;
} __gmp_randstate_struct;
typedef __gmp_randstate_struct gmp_randstate_t[1];

extern const char* const __gmp_version;
#define gmp_version __gmp_version

void __gmpz_init(mpz_ptr);
void __gmpz_clear(mpz_ptr);
void __gmpz_set_ui(mpz_ptr, unsigned long);
void __gmpz_set_si(mpz_ptr, long);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_sub_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_tdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_tdiv_r_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_mod(mpz_ptr, mpz_srcptr, mpz_srcptr);
int __gmpz_cmp(mpz_srcptr, mpz_srcptr);
int __gmpz_cmp_ui(mpz_srcptr, unsigned long);
unsigned long __gmpz_get_ui(mpz_srcptr);
char* __gmpz_get_str(char*, int, mpz_srcptr);
size_t __gmpz_sizeinbase(mpz_srcptr, int);
void __gmpz_urandomb(mpz_ptr, gmp_randstate_t, mp_bitcnt_t);
void* __gmpz_export(void*, size_t*, int, size_t, int, size_t, mpz_srcptr);
void __gmpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void*);
void __gmp_randinit_default(gmp_randstate_t);
void __gmp_randclear(gmp_randstate_t);
void __gmp_get_memory_functions(void* (**)(size_t), void* (**)(void*, size_t, size_t),
                                void (**)(void*, size_t));

#define mpz_init __gmpz_init
#define mpz_clear __gmpz_clear
#define mpz_set_ui __gmpz_set_ui
#define mpz_set_si __gmpz_set_si
#define mpz_mul __gmpz_mul
#define mpz_mul_2exp __gmpz_mul_2exp
#define mpz_add __gmpz_add
#define mpz_add_ui __gmpz_add_ui
#define mpz_sub __gmpz_sub
#define mpz_sub_ui __gmpz_sub_ui
#define mpz_tdiv_q_2exp __gmpz_tdiv_q_2exp
#define mpz_tdiv_r_2exp __gmpz_tdiv_r_2exp
#define mpz_mod __gmpz_mod
#define mpz_cmp __gmpz_cmp
#define mpz_cmp_ui __gmpz_cmp_ui
#define mpz_get_ui __gmpz_get_ui
#define mpz_get_str __gmpz_get_str
#define mpz_sizeinbase __gmpz_sizeinbase
#define mpz_urandomb __gmpz_urandomb
#define mpz_export __gmpz_export
#define mpz_import __gmpz_import
#define gmp_randinit_default __gmp_randinit_default
#define gmp_randclear __gmp_randclear
#define mp_get_memory_functions __gmp_get_memory_functions

#ifdef __cplusplus
}
#endif

#endif
