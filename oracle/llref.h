/* THE ORACLE: a CPU restatement of the reference's Lucas-Lehmer path, used only as the checker.
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference arm may load it, and only to check or to time the CPU side. The product
 * (mersenneprime_python_cpp_gmp_benchmark_b200/) never links, loads or calls anything here.
 *
 * What it restates (reference = wadeghcp/MersennePrime_Python_CPP_GMP_BenchMark):
 *   orc_ll_gmp        lucaslehmer.cpp:29-58    GMP squaring, -2, shift-and-add reduction mod 2^p-1
 *   orc_rebuild       lucaslehmer.cpp:312-323  digits -> exact residue mod 2^p-1 (also ll_ntt.cu:238-252)
 *   orc_fft_length    lucaslehmer.cpp:244-254  smallest {1,3,5}*2^k length at <= max_bpw bits/word
 *   orc_ibdwt         lucaslehmer.cpp:257-329  the FP64 IBDWT engine, on the oracle's own FFT (cfft.c)
 *   orc_gl_*          ll_ntt.cu:38-61          Goldilocks field arithmetic (here with 128-bit integers)
 *   orc_ntt_length    ll_ntt.cu:172-180        NTT exactness bound and length choice
 *   orc_ntt_tables    ll_ntt.cu:182-195        roots of unity and the N-th root of 2
 *   orc_ntt           ll_ntt.cu:74-167         the integer IBDWT loop, run on the CPU
 *
 * GMP (6.3.0, the version the reference's README measured; the reference itself pins none) is a
 * third-party dependency; its mpz API is reached through shim/gmp.h.
 *
 * Parity is pinned: tests/golden/ holds vectors produced by the reference's own GMP engine
 * (compiled unchanged from its sources into oracle/_ref/) and the reference README's published
 * interim residue; tests/test_oracle.py checks this file against all of them. */
#ifndef ORACLE_LLREF_H
#define ORACLE_LLREF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* s_k after `iters` squarings (iters == 0: the full p-2) from s_0 = 4, modulo 2^p - 1.
 * Returns 1 when the residue is 0 (for the full run: M_p prime), else 0. p < 2 -> 0, p == 2 -> 1,
 * even p -> 0 (no iterations run, residue reported as 0). words: ceil(p/64) little-endian limbs. */
int orc_ll_gmp(uint64_t p, uint64_t iters, uint64_t* res64, uint64_t* words, size_t nwords);
/* res64 after every `every` iterations up to `iters`: out[i] = res64 after (i+1)*every squarings. */
int orc_ll_gmp_trace(uint64_t p, uint64_t iters, uint64_t every, uint64_t* out, size_t nout);

/* sum_j digits[j] * 2^ceil(jp/N) mod 2^p - 1 (exact). */
int orc_rebuild(uint64_t p, uint64_t N, const int64_t* digits, uint64_t* res64, uint64_t* words,
                size_t nwords);

uint64_t orc_fft_length(uint64_t p, double max_bpw);
/* Returns 1 prime / 0 composite / -1 when the round-off ever exceeds abort_err. N == 0 picks
 * orc_fft_length(p, 18). digits_out (N entries) may be NULL. */
int orc_ibdwt(uint64_t p, uint64_t N, uint64_t iters, double abort_err, double* maxerr,
              int64_t* digits_out, uint64_t* res64, uint64_t* words, size_t nwords);

uint64_t orc_gl_add(uint64_t a, uint64_t b);
uint64_t orc_gl_sub(uint64_t a, uint64_t b);
uint64_t orc_gl_mul(uint64_t a, uint64_t b);
uint64_t orc_gl_pow(uint64_t a, uint64_t e);
int orc_ntt_max_bits(uint64_t N);
uint64_t orc_ntt_length(uint64_t p);
/* omega = primitive N-th root of unity, root2 = an N-th root of 2, invN = N^-1 (all in GF(q)). */
int orc_ntt_tables(uint64_t N, uint64_t* omega, uint64_t* root2, uint64_t* invN);
int orc_ntt(uint64_t p, uint64_t N, uint64_t iters, int64_t* digits_out, uint64_t* res64,
            uint64_t* words, size_t nwords);

#ifdef __cplusplus
}
#endif

#endif
