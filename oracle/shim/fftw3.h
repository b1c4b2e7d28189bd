/* Declaration header for the subset of the FFTW3 API that the reference's FFT engine calls
 * (plan, allocate, execute r2c / c2r). TEST INFRASTRUCTURE ONLY: FFTW3 is not installed on these
 * machines, so the reference's lucaslehmer.cpp is compiled unchanged against this header and the
 * implementation in fftw_shim.c, which runs the oracle's own mixed-radix FFT (oracle/cfft.c).
 * Anything timed through it is the reference's engine on the oracle's FFT, not on FFTW. */
#ifndef ORACLE_SHIM_FFTW3_H
#define ORACLE_SHIM_FFTW3_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_ESTIMATE (1U << 6)

double* fftw_alloc_real(size_t n);
fftw_complex* fftw_alloc_complex(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_dft_r2c_1d(int n, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex* in, double* out, unsigned flags);
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif
