/* FFTW3-API shim over the oracle's own FFT (test infrastructure only; see fftw3.h). Plans are
 * immutable after creation and every execute call uses its own thread-local scratch, so concurrent
 * executes from many threads are safe, as the reference's engine assumes. */
#include "fftw3.h"

#include <stdlib.h>

#include "../cfft.h"

struct fftw_plan_s {
    int n;
    cfft_plan* half;
};

static _Thread_local double* t_scratch = NULL;
static _Thread_local size_t t_scratch_n = 0;

static double* scratch_for(size_t n) {
    if (t_scratch_n < n) {
        free(t_scratch);
        t_scratch = (double*)malloc(sizeof(double) * 2 * n);
        t_scratch_n = n;
    }
    return t_scratch;
}

double* fftw_alloc_real(size_t n) { return (double*)aligned_alloc(64, ((n * sizeof(double) + 63) / 64) * 64); }
fftw_complex* fftw_alloc_complex(size_t n) {
    return (fftw_complex*)aligned_alloc(64, ((n * sizeof(fftw_complex) + 63) / 64) * 64);
}
void fftw_free(void* p) { free(p); }

static fftw_plan make(int n) {
    if (n < 2 || (n & 1)) return NULL;
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->n = n;
    p->half = cfft_plan_new((size_t)n / 2);
    if (!p->half) {
        free(p);
        return NULL;
    }
    return p;
}

fftw_plan fftw_plan_dft_r2c_1d(int n, double* in, fftw_complex* out, unsigned flags) {
    (void)in; (void)out; (void)flags;
    return make(n);
}
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex* in, double* out, unsigned flags) {
    (void)in; (void)out; (void)flags;
    return make(n);
}
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out) {
    rfft_r2c(p->half, in, (double*)out, scratch_for((size_t)p->n));
}
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out) {
    rfft_c2r(p->half, (const double*)in, out, scratch_for((size_t)p->n));
}
void fftw_destroy_plan(fftw_plan p) {
    if (!p) return;
    cfft_plan_free(p->half);
    free(p);
}
