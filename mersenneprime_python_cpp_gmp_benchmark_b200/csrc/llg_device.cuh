// Device-side building blocks shared by the Lucas-Lehmer kernels (sm_100a):
//   * complex FP64 arithmetic on double2 and fixed-radix in-register DFTs (2, 4, 8, 16 points);
//   * twiddles from a quarter-wave table (one load and a rotation by a power of -i);
//   * round-to-nearest with the 1.5*2^52 shifter, which also yields the integer in the low bits;
//   * the balanced-digit carry step of the irrational-base DWT.
//
// The arithmetic follows the IBDWT of the reference's FFT engine (lucaslehmer.cpp:257-311):
// digits x_j in a variable base of b_j = ceil((j+1)p/N) - ceil(jp/N) bits, weights
// a_j = 2^(ceil(jp/N) - jp/N), a cyclic convolution of the weighted digits, unweight, round,
// balanced carry with the "- 2" folded into digit 0 and the top carry wrapping into digit 0.
#pragma once

#include <cstdint>

namespace llg {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }
// a * (-i) and a * (+i)
__device__ __forceinline__ double2 mul_mi(double2 a) { return make_double2(a.y, -a.x); }
__device__ __forceinline__ double2 mul_pi(double2 a) { return make_double2(-a.y, a.x); }

// Multiply by e^{-2 pi i k / R} (INV=false) or e^{+2 pi i k / R} (INV=true) for a compile-time
// k / R with R in {2, 4, 8, 16}. Special angles use adds only; the rest use exact constants.
template <int R, int K, bool INV>
__device__ __forceinline__ double2 rot(double2 a) {
    constexpr int k = ((K % R) + R) % R;
    constexpr int k16 = k * (16 / R);  // angle in units of 2*pi/16
    if constexpr (k16 == 0) return a;
    constexpr double C1 = 0.92387953251128675613;  // cos(pi/8)
    constexpr double S1 = 0.38268343236508977173;  // sin(pi/8)
    constexpr double H = 0.70710678118654752440;   // cos(pi/4)
    // e^{-2 pi i k16/16} = cos(t) - i sin(t), t = k16*pi/8
    constexpr double cs[16] = {1, C1, H, S1, 0, -S1, -H, -C1, -1, -C1, -H, -S1, 0, S1, H, C1};
    constexpr double sn[16] = {0, S1, H, C1, 1, C1, H, S1, 0, -S1, -H, -C1, -1, -C1, -H, -S1};
    constexpr double c = cs[k16];
    constexpr double s = INV ? -sn[k16] : sn[k16];  // multiply by (c - i s)
    if constexpr (k16 == 4) return INV ? mul_pi(a) : mul_mi(a);
    if constexpr (k16 == 8) return make_double2(-a.x, -a.y);
    if constexpr (k16 == 12) return INV ? mul_mi(a) : mul_pi(a);
    if constexpr (k16 == 2 || k16 == 6 || k16 == 10 || k16 == 14) {
        // (a.x + i a.y)(c - i s) with |c| = |s| = H
        return make_double2(H * ((c > 0 ? a.x : -a.x) + (s > 0 ? a.y : -a.y)),
                            H * ((c > 0 ? a.y : -a.y) - (s > 0 ? a.x : -a.x)));
    }
    return make_double2(fma(a.x, c, a.y * s), fma(a.y, c, -a.x * s));
}

// rot<16, k16, INV> for a k16 known only after unrolling (the switch folds away).
template <bool INV>
__device__ __forceinline__ double2 rot16_k(double2 a, int k16) {
    switch (k16 & 15) {
        case 0: return a;
        case 1: return rot<16, 1, INV>(a);
        case 2: return rot<16, 2, INV>(a);
        case 3: return rot<16, 3, INV>(a);
        case 4: return rot<16, 4, INV>(a);
        case 5: return rot<16, 5, INV>(a);
        case 6: return rot<16, 6, INV>(a);
        case 7: return rot<16, 7, INV>(a);
        case 8: return rot<16, 8, INV>(a);
        case 9: return rot<16, 9, INV>(a);
        case 10: return rot<16, 10, INV>(a);
        case 11: return rot<16, 11, INV>(a);
        case 12: return rot<16, 12, INV>(a);
        case 13: return rot<16, 13, INV>(a);
        case 14: return rot<16, 14, INV>(a);
        default: return rot<16, 15, INV>(a);
    }
}
// Multiply by e^{-2 pi i k / R} (INV: e^{+2 pi i k / R}), R in {1, 2, 4, 8, 16}.
template <int R, bool INV>
__device__ __forceinline__ double2 rot_k(double2 a, int k) {
    if constexpr (R == 1) return a;
    else return rot16_k<INV>(a, (k & (R - 1)) * (16 / R));
}

// In-register DFT of R points, natural order in and out:
//   X_k = sum_n x_n e^{-+2 pi i nk/R}   (sign - for the forward transform, + for INV; unscaled).
template <int R, bool INV>
struct Dft;

template <bool INV>
struct Dft<1, INV> {
    __device__ __forceinline__ static void run(double2*) {}
};

template <bool INV>
struct Dft<2, INV> {
    __device__ __forceinline__ static void run(double2* v) {
        double2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <bool INV>
struct Dft<4, INV> {
    __device__ __forceinline__ static void run(double2* v) {
        double2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        double2 b0 = cadd(v[1], v[3]), b1 = csub(v[1], v[3]);
        b1 = INV ? mul_pi(b1) : mul_mi(b1);
        v[0] = cadd(a0, b0);
        v[2] = csub(a0, b0);
        v[1] = cadd(a1, b1);
        v[3] = csub(a1, b1);
    }
};

// R = R1 * R2 split (decimation in frequency on the register array):
//   X[k1 + R1 k2] = sum_{n2} w_{R2}^{n2 k2} w_R^{n2 k1} sum_{n1} x[n1 R2 + n2] w_{R1}^{n1 k1}
template <int R1, int R2, bool INV>
struct DftSplit {
    static constexpr int R = R1 * R2;
    template <int N2, int K1>
    __device__ __forceinline__ static void twiddle_all(double2 (&a)[R1][R2]) {
        if constexpr (N2 < R2) {
            if constexpr (K1 < R1) {
                a[K1][N2] = rot<R, N2 * K1, INV>(a[K1][N2]);
                twiddle_all<N2, K1 + 1>(a);
            } else {
                twiddle_all<N2 + 1, 0>(a);
            }
        }
    }
    __device__ __forceinline__ static void run(double2* v) {
        double2 a[R1][R2];
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) {
            double2 col[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; ++n1) col[n1] = v[n1 * R2 + n2];
            Dft<R1, INV>::run(col);
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) a[k1][n2] = col[k1];
        }
        twiddle_all<0, 0>(a);
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) {
            Dft<R2, INV>::run(a[k1]);
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = a[k1][k2];
        }
    }
};

template <bool INV>
struct Dft<8, INV> {
    __device__ __forceinline__ static void run(double2* v) { DftSplit<2, 4, INV>::run(v); }
};
template <bool INV>
struct Dft<16, INV> {
    __device__ __forceinline__ static void run(double2* v) { DftSplit<4, 4, INV>::run(v); }
};

// Quarter-wave tables are stored padded: entry r at qpad(r) = r + r/8, so the strided indices of
// the radix passes (multiples of 16 and of small odd numbers) spread over the shared-memory banks.
__host__ __device__ constexpr uint32_t qpad(uint32_t r) { return r + (r >> 3); }
__host__ __device__ constexpr uint32_t qpad_len(uint32_t qm) { return qm + (qm >> 3) + 1; }
// The same quarter-wave table spread further, entry r at r + r/8 + r/64: the whole-test kernel's
// twiddle reads at index n2 k1 (8 lanes of a quarter warp, strides k1 and 16 k1) and its
// digit-reversed real-FFT twiddles then land in more of the 8 bank groups of 16-byte slots.
__host__ __device__ constexpr uint32_t qpad_s(uint32_t r) { return r + (r >> 3) + (r >> 6); }
__host__ __device__ constexpr uint32_t qpad_s_len(uint32_t qm) { return qm + (qm >> 3) + (qm >> 6) + 1; }
static_assert(qpad_s(255) < qpad_s_len(256) && qpad_s(1023) < qpad_s_len(1024) && qpad_s(4095) < qpad_s_len(4096),
              "spread quarter table length");

// Twiddle e^{-2 pi i x / M} (conjugated when inv) from a padded quarter-wave table
// q[qpad(r)] = e^{-2 pi i r / M}, r < M/4.  x in [0, M).
// SPREAD: the table is in the qpad_s layout.
template <int LOG_M, bool SPREAD = false>
__device__ __forceinline__ double2 twiddle(const double2* __restrict__ q, uint32_t x, bool inv) {
    constexpr uint32_t QM = (1u << LOG_M) / 4;
    const uint32_t quad = (x / QM) & 3u;
    double2 w = q[SPREAD ? qpad_s(x % QM) : qpad(x % QM)];
    // rotate by (-i)^quad
    double2 r;
    switch (quad) {
        case 0: r = w; break;
        case 1: r = make_double2(w.y, -w.x); break;
        case 2: r = make_double2(-w.x, -w.y); break;
        default: r = make_double2(-w.y, w.x); break;
    }
    return inv ? conj2(r) : r;
}

// Round to nearest even with the 1.5*2^52 shifter (valid for |v| < 2^51): returns the rounded
// double and the same integer as int64.
__device__ __forceinline__ double round_shift(double v, long long& iv) {
    constexpr double SH = 6755399441055744.0;  // 1.5 * 2^52
    const double t = __dadd_rn(v, SH);
    iv = __double_as_longlong(t) - 0x4338000000000000LL;
    return __dsub_rn(t, SH);
}

// Exact conversion of a small signed integer (|x| < 2^51) to double by the same shifter.
__device__ __forceinline__ double i2d_shift(long long x) {
    constexpr double SH = 6755399441055744.0;
    return __dsub_rn(__longlong_as_double(x + 0x4338000000000000LL), SH);
}

// Programmatic dependent launch (griddepcontrol, sm_90 and later): let the next kernel of the
// stream launch once every block of this one has executed it, and wait until the previous kernel
// has completed with its memory visible. Both are no-ops in a launch without the programmatic
// stream serialisation attribute.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait_previous() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Asynchronous global -> shared copies (cp.async, completed by cp_async_wait_all, then a barrier
// before other threads read the data).
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async sizes");
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(s), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// 2^e as a double (normal range).
__device__ __forceinline__ double pow2(int e) { return __longlong_as_double((long long)(1023 + e) << 52); }

// Balanced split of an integer-valued double: v = x + c 2^b with |x| <= 2^(b-1) (ties to even),
// c and x exact for |v| < 2^51; inv = 2^-b, pw = 2^b. The FP64 form of the reference's carry step
// (lucaslehmer.cpp:299-303: c = floor((v + 2^(b-1)) / 2^b)); the two differ only at ties, and
// either representation of the residue is exact.
__device__ __forceinline__ double dsplit(double v, double inv, double pw, double& c) {
    constexpr double SH = 6755399441055744.0;  // 1.5 * 2^52: adding it rounds to an integer
    c = __dsub_rn(__fma_rn(v, inv, SH), SH);
    return __fma_rn(-c, pw, v);
}

// dsplit with digit size e bits: 2^e and 2^-e built from the exponent field (few live registers).
__device__ __forceinline__ double dsplit_e(double v, int e, double& c) {
    const double pw = __hiloint2double((1023 + e) << 20, 0), inv = __hiloint2double((1023 - e) << 20, 0);
    return dsplit(v, inv, pw, c);
}

// An integer-valued double with |x| < 2^31 as int32 (the low word of x + 1.5 * 2^52).
__device__ __forceinline__ int d2i_exact(double x) { return __double2loint(__dadd_rn(x, 6755399441055744.0)); }

// One balanced-digit step: v = x + carry_in; returns the digit in [-2^(b-1), 2^(b-1)) and sets
// carry = floor((v + 2^(b-1)) / 2^b)  (lucaslehmer.cpp:299-303).
__device__ __forceinline__ long long balance(long long v, int b, long long& carry) {
    const long long c = (v + (1LL << (b - 1))) >> b;
    carry = c;
    return v - (c << b);
}

}  // namespace llg
