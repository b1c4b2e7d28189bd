/* Oracle-side CPU FFT (test infrastructure only; see cfft.h). A textbook recursive mixed-radix
 * decimation-in-time complex FFT with radix 4, 2, 3 and 5 butterflies, plus the standard
 * "two real halves in one complex transform" real-input / real-output wrappers. */
#include "cfft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct cfft_plan {
    size_t n;
    double* tw;  /* omega_n^k = e^{-2 pi i k/n}, k < n (interleaved) */
    double* tw2; /* omega_{2n}^k, k < n: the post-processing twiddles of a 2n-point real FFT */
};

static void fill(double* t, size_t period, size_t count) {
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (size_t k = 0; k < count; ++k) {
        long double a = -two_pi * (long double)k / (long double)period;
        t[2 * k] = (double)cosl(a);
        t[2 * k + 1] = (double)sinl(a);
    }
}

cfft_plan* cfft_plan_new(size_t n) {
    size_t m = n;
    if (n == 0) return NULL;
    while (m % 2 == 0) m /= 2;
    while (m % 3 == 0) m /= 3;
    while (m % 5 == 0) m /= 5;
    if (m != 1) return NULL;
    cfft_plan* p = (cfft_plan*)calloc(1, sizeof(cfft_plan));
    p->n = n;
    p->tw = (double*)malloc(sizeof(double) * 2 * n);
    p->tw2 = (double*)malloc(sizeof(double) * 2 * n);
    fill(p->tw, n, n);
    fill(p->tw2, 2 * n, n);
    return p;
}

void cfft_plan_free(cfft_plan* p) {
    if (!p) return;
    free(p->tw);
    free(p->tw2);
    free(p);
}

size_t cfft_size(const cfft_plan* p) { return p->n; }

/* out[k] = sum_j in[j*is] * w^{jk}, w = omega_n (conjugated when sign > 0). ts = plan->n / n. */
static void rec(const cfft_plan* P, const double* in, size_t is, double* out, size_t n, size_t ts,
                int sign) {
    if (n == 1) {
        out[0] = in[0];
        out[1] = in[1];
        return;
    }
    const size_t r = (n % 4 == 0) ? 4 : (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : 5;
    const size_t m = n / r;
    for (size_t q = 0; q < r; ++q) rec(P, in + 2 * q * is, is * r, out + 2 * q * m, m, ts * r, sign);
    const double s = (sign > 0) ? 1.0 : -1.0; /* sign of the imaginary part of w */
    for (size_t k = 0; k < m; ++k) {
        double tr[5], ti[5];
        for (size_t q = 0; q < r; ++q) {
            const double xr = out[2 * (q * m + k)], xi = out[2 * (q * m + k) + 1];
            const double* w = P->tw + 2 * (q * k * ts);
            const double wr = w[0], wi = (sign > 0) ? -w[1] : w[1];
            tr[q] = xr * wr - xi * wi;
            ti[q] = xr * wi + xi * wr;
        }
        double* o0 = out + 2 * k;
        if (r == 2) {
            o0[0] = tr[0] + tr[1];
            o0[1] = ti[0] + ti[1];
            o0[2 * m] = tr[0] - tr[1];
            o0[2 * m + 1] = ti[0] - ti[1];
        } else if (r == 4) {
            /* w4 = e^{sign i pi/2} = s*i; (x)(s i) = (-s xi, s xr) */
            const double a0r = tr[0] + tr[2], a0i = ti[0] + ti[2];
            const double a1r = tr[0] - tr[2], a1i = ti[0] - ti[2];
            const double b0r = tr[1] + tr[3], b0i = ti[1] + ti[3];
            const double dr = tr[1] - tr[3], di = ti[1] - ti[3];
            const double b1r = -s * di, b1i = s * dr;
            o0[0] = a0r + b0r;
            o0[1] = a0i + b0i;
            o0[2 * m] = a1r + b1r;
            o0[2 * m + 1] = a1i + b1i;
            o0[4 * m] = a0r - b0r;
            o0[4 * m + 1] = a0i - b0i;
            o0[6 * m] = a1r - b1r;
            o0[6 * m + 1] = a1i - b1i;
        } else {
            for (size_t u = 0; u < r; ++u) {
                double accr = 0.0, acci = 0.0;
                for (size_t q = 0; q < r; ++q) {
                    const double* w = P->tw + 2 * (((q * u) % r) * m * ts);
                    const double wr = w[0], wi = (sign > 0) ? -w[1] : w[1];
                    accr += tr[q] * wr - ti[q] * wi;
                    acci += tr[q] * wi + ti[q] * wr;
                }
                o0[2 * u * m] = accr;
                o0[2 * u * m + 1] = acci;
            }
        }
    }
}

void cfft_exec(const cfft_plan* p, double* data, int sign, double* scratch) {
    rec(p, data, 1, scratch, p->n, 1, sign);
    memcpy(data, scratch, sizeof(double) * 2 * p->n);
}

void rfft_r2c(const cfft_plan* P, const double* in, double* out, double* scratch) {
    const size_t h = P->n;
    memcpy(out, in, sizeof(double) * 2 * h);
    cfft_exec(P, out, -1, scratch);
    /* Y_k = (Z_k + conj Z_{h-k})/2 + w^k (Z_k - conj Z_{h-k})/(2i),  w = omega_{2h} */
    const double z0r = out[0], z0i = out[1];
    for (size_t k = 1; 2 * k <= h; ++k) {
        const size_t j = h - k;
        const double ar = out[2 * k], ai = out[2 * k + 1];
        const double br = out[2 * j], bi = out[2 * j + 1];
        /* k side */
        double er = 0.5 * (ar + br), ei = 0.5 * (ai - bi);       /* (Z_k + conj Z_j)/2 */
        double orr = 0.5 * (ai + bi), oi = -0.5 * (ar - br);      /* (Z_k - conj Z_j)/(2i) */
        const double* w = P->tw2 + 2 * k;
        double yr = er + (w[0] * orr - w[1] * oi), yi = ei + (w[0] * oi + w[1] * orr);
        /* j side: (Z_j + conj Z_k)/2 + w^j (Z_j - conj Z_k)/(2i) */
        double fr = 0.5 * (br + ar), fi = 0.5 * (bi - ai);
        double pr = 0.5 * (bi + ai), pi = -0.5 * (br - ar);
        const double* v = P->tw2 + 2 * j;
        double xr = fr + (v[0] * pr - v[1] * pi), xi = fi + (v[0] * pi + v[1] * pr);
        out[2 * k] = yr;
        out[2 * k + 1] = yi;
        out[2 * j] = xr;
        out[2 * j + 1] = xi;
    }
    out[0] = z0r + z0i;
    out[1] = 0.0;
    out[2 * h] = z0r - z0i;
    out[2 * h + 1] = 0.0;
}

void rfft_c2r(const cfft_plan* P, const double* in, double* out, double* scratch) {
    const size_t h = P->n;
    /* Z'_k = (Y_k + Y_{k+h}) + i (Y_k - Y_{k+h}) e^{+2 pi i k/(2h)},  Y_{k+h} = conj Y_{h-k} */
    for (size_t k = 0; k < h; ++k) {
        const size_t j = h - k;
        double ar = in[2 * k], ai = in[2 * k + 1];
        double br = in[2 * j], bi = -in[2 * j + 1];
        if (k == 0) {
            ai = 0.0;
            bi = 0.0;
        }
        if (j == h) bi = 0.0;
        const double sr = ar + br, si = ai + bi;
        const double dr = ar - br, di = ai - bi;
        const double wr = P->tw2[2 * k], wi = -P->tw2[2 * k + 1]; /* conj: e^{+...} */
        const double tr = dr * wr - di * wi, ti = dr * wi + di * wr;
        out[2 * k] = sr - ti; /* + i * (tr + i ti) */
        out[2 * k + 1] = si + tr;
    }
    cfft_exec(P, out, +1, scratch);
}
