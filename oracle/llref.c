/* THE ORACLE (test infrastructure only): CPU restatement of the reference's Lucas-Lehmer path.
 * See llref.h for what each function restates (file:line in the reference) and who may call it. */
#include "llref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "cfft.h"
#include "shim/gmp.h"

typedef unsigned __int128 u128;

/* ---- GMP engine: lucaslehmer.cpp:29-58 ------------------------------------------------------ */

static void export_words(const mpz_t s, uint64_t* words, size_t nwords) {
    if (!words) return;
    memset(words, 0, nwords * sizeof(uint64_t));
    size_t cnt = 0;
    size_t need = (mpz_sizeinbase(s, 2) + 63) / 64;
    if (mpz_cmp_ui(s, 0) == 0) return;
    if (need > nwords) return; /* caller sized it wrong; leave zeros */
    mpz_export(words, &cnt, -1, sizeof(uint64_t), 0, 0, s);
}

/* One LL step: s = s^2 - 2 mod M, with M = 2^p - 1, by the shift-and-add reduction. */
static void ll_step(mpz_t s, const mpz_t M, uint64_t p, mpz_t hi) {
    mpz_mul(s, s, s);
    mpz_sub_ui(s, s, 2);
    mpz_tdiv_q_2exp(hi, s, p);
    mpz_tdiv_r_2exp(s, s, p);
    mpz_add(s, s, hi);
    if (mpz_cmp(s, M) >= 0) mpz_sub(s, s, M);
}

int orc_ll_gmp(uint64_t p, uint64_t iters, uint64_t* res64, uint64_t* words, size_t nwords) {
    if (res64) *res64 = 0;
    if (words) memset(words, 0, nwords * sizeof(uint64_t));
    if (p < 2) return 0;
    if (p == 2) return 1;
    if (p % 2 == 0) return 0;
    mpz_t M, s, hi;
    mpz_init(M);
    mpz_init(s);
    mpz_init(hi);
    mpz_set_ui(M, 1);
    mpz_mul_2exp(M, M, p);
    mpz_sub_ui(M, M, 1);
    mpz_set_ui(s, 4);
    for (uint64_t i = 0; i + 2 < p && (!iters || i < iters); ++i) ll_step(s, M, p, hi);
    if (res64) *res64 = mpz_get_ui(s);
    export_words(s, words, nwords);
    int prime = mpz_cmp_ui(s, 0) == 0;
    mpz_clear(M);
    mpz_clear(s);
    mpz_clear(hi);
    return prime;
}

int orc_ll_gmp_trace(uint64_t p, uint64_t iters, uint64_t every, uint64_t* out, size_t nout) {
    if (p < 3 || (p % 2 == 0) || every == 0) return -1;
    mpz_t M, s, hi;
    mpz_init(M);
    mpz_init(s);
    mpz_init(hi);
    mpz_set_ui(M, 1);
    mpz_mul_2exp(M, M, p);
    mpz_sub_ui(M, M, 1);
    mpz_set_ui(s, 4);
    size_t k = 0;
    for (uint64_t i = 0; i + 2 < p && i < iters; ++i) {
        ll_step(s, M, p, hi);
        if ((i + 1) % every == 0 && k < nout) out[k++] = mpz_get_ui(s);
    }
    mpz_clear(M);
    mpz_clear(s);
    mpz_clear(hi);
    return (int)k;
}

/* ---- residue rebuild: lucaslehmer.cpp:312-323 ----------------------------------------------- */

static uint64_t ceil_div_u(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a + b - 1) / b); }
static uint64_t ceil_jp_n(uint64_t j, uint64_t p, uint64_t N) {
    return (uint64_t)(((u128)j * p + N - 1) / N);
}

int orc_rebuild(uint64_t p, uint64_t N, const int64_t* digits, uint64_t* res64, uint64_t* words,
                size_t nwords) {
    mpz_t M, s, t;
    mpz_init(M);
    mpz_init(s);
    mpz_init(t);
    mpz_set_ui(M, 1);
    mpz_mul_2exp(M, M, p);
    mpz_sub_ui(M, M, 1);
    for (uint64_t j = 0; j < N; ++j) {
        if (!digits[j]) continue;
        mpz_set_si(t, (long)digits[j]);
        mpz_mul_2exp(t, t, ceil_jp_n(j, p, N));
        mpz_add(s, s, t);
    }
    mpz_mod(s, s, M);
    if (res64) *res64 = mpz_get_ui(s);
    export_words(s, words, nwords);
    int zero = mpz_cmp_ui(s, 0) == 0;
    mpz_clear(M);
    mpz_clear(s);
    mpz_clear(t);
    return zero;
}

/* ---- FP64 IBDWT engine: lucaslehmer.cpp:244-335 --------------------------------------------- */

uint64_t orc_fft_length(uint64_t p, double max_bpw) {
    if (max_bpw <= 0) max_bpw = 18.0;
    uint64_t best = 0;
    const uint64_t ms[3] = {1, 3, 5};
    for (int i = 0; i < 3; ++i)
        for (uint64_t N = ms[i] * 16; N < ((uint64_t)1 << 40); N <<= 1)
            if ((double)p / (double)N <= max_bpw) {
                if (!best || N < best) best = N;
                break;
            }
    return best;
}

int orc_ibdwt(uint64_t p, uint64_t N, uint64_t iters, double abort_err, double* maxerr_out,
              int64_t* digits_out, uint64_t* res64, uint64_t* words, size_t nwords) {
    if (res64) *res64 = 0;
    if (maxerr_out) *maxerr_out = 0.0;
    if (p < 3 || (p % 2 == 0)) return -1;
    if (N == 0) N = orc_fft_length(p, 18.0);
    if (N < 4 || (N & 1)) return -1;
    cfft_plan* plan = cfft_plan_new(N / 2);
    if (!plan) return -1;
    int* bits = (int*)malloc(sizeof(int) * N);
    double* w = (double*)malloc(sizeof(double) * N);
    double* winv = (double*)malloc(sizeof(double) * N);
    int64_t* x = (int64_t*)calloc(N, sizeof(int64_t));
    double* y = (double*)malloc(sizeof(double) * N);
    double* Y = (double*)malloc(sizeof(double) * (N + 2));
    double* scratch = (double*)malloc(sizeof(double) * 2 * N);
    for (uint64_t j = 0; j < N; ++j) {
        uint64_t lo = ceil_jp_n(j, p, N), hi = ceil_jp_n(j + 1, p, N);
        bits[j] = (int)(hi - lo);
        long double frac = (long double)(uint64_t)((u128)lo * N - (u128)j * p) / (long double)N;
        w[j] = (double)exp2l(frac);
        winv[j] = (double)(1.0L / (exp2l(frac) * (long double)N));
    }
    x[0] = 4;
    double maxerr = 0.0;
    int verdict = -1;
    for (uint64_t it = 0; it + 2 < p && (!iters || it < iters); ++it) {
        for (uint64_t j = 0; j < N; ++j) y[j] = (double)x[j] * w[j];
        rfft_r2c(plan, y, Y, scratch);
        for (uint64_t k = 0; k <= N / 2; ++k) {
            double re = Y[2 * k], im = Y[2 * k + 1];
            Y[2 * k] = re * re - im * im;
            Y[2 * k + 1] = 2.0 * re * im;
        }
        rfft_c2r(plan, Y, y, scratch);
        double err = 0.0;
        for (uint64_t j = 0; j < N; ++j) {
            double v = y[j] * winv[j], r = nearbyint(v);
            double e = fabs(v - r);
            if (e > err) err = e;
            y[j] = r;
        }
        if (err > maxerr) maxerr = err;
        if (err > abort_err) goto done;
        int64_t carry = -2;
        for (uint64_t j = 0; j < N; ++j) {
            int64_t v = (int64_t)y[j] + carry;
            int b = bits[j];
            carry = (v + ((int64_t)1 << (b - 1))) >> b;
            x[j] = v - (carry << b);
        }
        while (carry) {
            for (uint64_t j = 0; j < N && carry; ++j) {
                int64_t v = x[j] + carry;
                int b = bits[j];
                carry = (v + ((int64_t)1 << (b - 1))) >> b;
                x[j] = v - (carry << b);
            }
        }
    }
    verdict = orc_rebuild(p, N, x, res64, words, nwords);
    if (digits_out) memcpy(digits_out, x, sizeof(int64_t) * N);
done:
    if (maxerr_out) *maxerr_out = maxerr;
    cfft_plan_free(plan);
    free(bits);
    free(w);
    free(winv);
    free(x);
    free(y);
    free(Y);
    free(scratch);
    return verdict;
}

/* ---- Goldilocks NTT engine: ll_ntt.cu:38-195 ------------------------------------------------ */

static const uint64_t GL_Q = 0xFFFFFFFF00000001ull;

uint64_t orc_gl_add(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a + b) % GL_Q); }
uint64_t orc_gl_sub(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a + GL_Q - b) % GL_Q); }
uint64_t orc_gl_mul(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) % GL_Q); }
uint64_t orc_gl_pow(uint64_t a, uint64_t e) {
    uint64_t r = 1;
    a %= GL_Q;
    while (e) {
        if (e & 1) r = orc_gl_mul(r, a);
        a = orc_gl_mul(a, a);
        e >>= 1;
    }
    return r;
}

int orc_ntt_max_bits(uint64_t N) {
    int l = 0;
    while (((uint64_t)1 << l) < N) ++l;
    return (63 - l) / 2;
}

uint64_t orc_ntt_length(uint64_t p) {
    for (uint64_t N = 64; N <= 8192; N <<= 1)
        if (ceil_div_u(p, N) <= (uint64_t)orc_ntt_max_bits(N)) return N;
    return 0;
}

int orc_ntt_tables(uint64_t N, uint64_t* omega, uint64_t* root2, uint64_t* invN) {
    if (N == 0 || (N & (N - 1)) || N > ((uint64_t)1 << 26)) return -1;
    const uint64_t g = 7;
    *omega = orc_gl_pow(g, (GL_Q - 1) / N);
    uint64_t om = orc_gl_pow(g, (GL_Q - 1) / (192 * N));
    uint64_t r192 = orc_gl_pow(om, N), pw = 1, s = 0;
    for (; s < 192; ++s) {
        if (pw == 2) break;
        pw = orc_gl_mul(pw, r192);
    }
    if (s == 192) return -1;
    *root2 = orc_gl_pow(om, s);
    *invN = orc_gl_pow(N % GL_Q, GL_Q - 2);
    return 0;
}

static void ntt_inplace(uint64_t* a, uint64_t N, uint64_t w) {
    /* iterative radix-2 DIT with bit reversal; w = primitive N-th root used for this direction */
    for (uint64_t i = 1, j = 0; i < N; ++i) {
        uint64_t bit = N >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            uint64_t t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
    for (uint64_t len = 2; len <= N; len <<= 1) {
        uint64_t wl = orc_gl_pow(w, N / len);
        for (uint64_t i = 0; i < N; i += len) {
            uint64_t wk = 1;
            for (uint64_t k = 0; k < len / 2; ++k) {
                uint64_t u = a[i + k], v = orc_gl_mul(a[i + k + len / 2], wk);
                a[i + k] = orc_gl_add(u, v);
                a[i + k + len / 2] = orc_gl_sub(u, v);
                wk = orc_gl_mul(wk, wl);
            }
        }
    }
}

int orc_ntt(uint64_t p, uint64_t N, uint64_t iters, int64_t* digits_out, uint64_t* res64,
            uint64_t* words, size_t nwords) {
    if (res64) *res64 = 0;
    if (p < 3 || (p % 2 == 0)) return -1;
    if (N == 0) N = orc_ntt_length(p);
    uint64_t omega, root2, invN;
    if (!N || orc_ntt_tables(N, &omega, &root2, &invN) != 0) return -1;
    const uint64_t omega_inv = orc_gl_pow(omega, GL_Q - 2);
    uint64_t* wgt = (uint64_t*)malloc(sizeof(uint64_t) * N);
    uint64_t* wgti = (uint64_t*)malloc(sizeof(uint64_t) * N);
    int* bits = (int*)malloc(sizeof(int) * N);
    int64_t* x = (int64_t*)calloc(N, sizeof(int64_t));
    uint64_t* s = (uint64_t*)malloc(sizeof(uint64_t) * N);
    for (uint64_t j = 0; j < N; ++j) {
        uint64_t c = ceil_jp_n(j, p, N);
        uint64_t e = (uint64_t)((u128)c * N - (u128)j * p);
        wgt[j] = orc_gl_pow(root2, e);
        wgti[j] = orc_gl_mul(orc_gl_pow(wgt[j], GL_Q - 2), invN);
        bits[j] = (int)(ceil_jp_n(j + 1, p, N) - c);
    }
    x[0] = 4;
    for (uint64_t it = 0; it + 2 < p && (!iters || it < iters); ++it) {
        for (uint64_t j = 0; j < N; ++j) {
            uint64_t f = x[j] < 0 ? GL_Q - (uint64_t)(-x[j]) : (uint64_t)x[j];
            s[j] = orc_gl_mul(f, wgt[j]);
        }
        ntt_inplace(s, N, omega);
        for (uint64_t j = 0; j < N; ++j) s[j] = orc_gl_mul(s[j], s[j]);
        ntt_inplace(s, N, omega_inv);
        int64_t carry = -2;
        for (uint64_t j = 0; j < N; ++j) {
            uint64_t v = orc_gl_mul(s[j], wgti[j]);
            int64_t sv = (v > (GL_Q >> 1)) ? -(int64_t)(GL_Q - v) : (int64_t)v;
            int b = bits[j];
            int64_t t = sv + carry;
            carry = (t + ((int64_t)1 << (b - 1))) >> b;
            x[j] = t - (carry << b);
        }
        while (carry) {
            for (uint64_t j = 0; j < N && carry; ++j) {
                int64_t t = x[j] + carry;
                int b = bits[j];
                carry = (t + ((int64_t)1 << (b - 1))) >> b;
                x[j] = t - (carry << b);
            }
        }
    }
    int verdict = orc_rebuild(p, N, x, res64, words, nwords);
    if (digits_out) memcpy(digits_out, x, sizeof(int64_t) * N);
    free(wgt);
    free(wgti);
    free(bits);
    free(x);
    free(s);
    return verdict;
}
