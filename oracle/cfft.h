/* Oracle-side CPU FFT: a plain mixed-radix (2, 3, 4, 5) complex FFT and the real-input /
 * real-output transforms built on it. TEST INFRASTRUCTURE ONLY (the checker's own transform, used
 * by the oracle's IBDWT restatement and by the FFTW3 API shim that lets the reference's FFT engine
 * compile where FFTW3 is absent). Not part of the product; nothing under the package links it.
 *
 * Conventions follow FFTW's: forward = sum x_j e^{-2 pi i jk/n}, inverse = sum X_k e^{+2 pi i jk/n},
 * both unnormalised. Twiddles are computed in long double and rounded once to double. */
#ifndef ORACLE_CFFT_H
#define ORACLE_CFFT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cfft_plan cfft_plan;

/* n must be of the form 2^a 3^b 5^c (n >= 1). */
cfft_plan* cfft_plan_new(size_t n);
void cfft_plan_free(cfft_plan* p);
size_t cfft_size(const cfft_plan* p);
/* data: n interleaved complex (re, im); sign = -1 forward, +1 inverse. scratch: 2n doubles. */
void cfft_exec(const cfft_plan* p, double* data, int sign, double* scratch);

/* Real transforms of even length n, built on an n/2-point complex plan (rp->n == n/2).
 * r2c: in[n] -> out[n/2+1] complex. c2r: in[n/2+1] complex -> out[n] (unnormalised; the imaginary
 * parts of bins 0 and n/2 are ignored). scratch: 2n doubles. */
void rfft_r2c(const cfft_plan* half, const double* in, double* out, double* scratch);
void rfft_c2r(const cfft_plan* half, const double* in, double* out, double* scratch);

#ifdef __cplusplus
}
#endif

#endif
