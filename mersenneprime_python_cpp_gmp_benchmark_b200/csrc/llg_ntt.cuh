// Arithmetic in GF(q), q = 2^64 - 2^32 + 1 ("Goldilocks"), and the in-register radix passes of
// the number-theoretic transforms (exact IBDWT; the reference's CUDA engine, cuda/ll_ntt.cu:38-61
// and 100-127, does the same field with radix-2 stages and a 128-bit-free u64 multiply).
//
//   * products: the 128-bit product is built from four 32 x 32-bit multiply-adds (mad.lo / mad.hi
//     with carry chains) and reduced with 2^64 == 2^32 - 1 and 2^96 == -1 (mod q);
//   * 2 has order 192, so every root of unity of order dividing 64 is a power of two: with the
//     primitive N-th roots w_N = 7^((q-1)/N) that the reference uses (cuda/ll_ntt.cu:187),
//     w_16 = 2^156, w_8 = 2^120, w_4 = 2^48, w_2 = 2^96 = -1. The twiddles inside a radix-16
//     butterfly are therefore shifts and a reduction, not products;
//   * values are kept canonical in [0, q).
#pragma once

#include <cstdint>

namespace llg {
namespace gl {

constexpr uint64_t Q = 0xFFFFFFFF00000001ull;
constexpr uint64_t EPS = 0xFFFFFFFFull;  // 2^64 mod q

// a + b for canonical a, b: the 65-bit sum with its carry c, and s + EPS with its carry; the
// result is s + EPS when either carried (a carry means a + b - 2^64 + EPS = a + b - q; a carry of
// s + EPS alone means s >= q), else s. 32-bit add-with-carry chains.
__device__ __forceinline__ uint64_t add(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("{\n\t.reg .u32 a0, a1, b0, b1, s0, s1, t0, t1, c, z;\n\t.reg .pred p;\n\t"
        "mov.u32 z, 0;\n\t"
        "mov.b64 {a0, a1}, %1;\n\t"
        "mov.b64 {b0, b1}, %2;\n\t"
        "add.cc.u32 s0, a0, b0;\n\t"
        "addc.cc.u32 s1, a1, b1;\n\t"
        "addc.u32 c, z, z;\n\t"
        "add.cc.u32 t0, s0, 0xFFFFFFFF;\n\t"
        "addc.cc.u32 t1, s1, z;\n\t"
        "addc.u32 c, c, z;\n\t"
        "setp.ne.u32 p, c, 0;\n\t"
        "selp.b32 s0, t0, s0, p;\n\t"
        "selp.b32 s1, t1, s1, p;\n\t"
        "mov.b64 %0, {s0, s1};\n\t}"
        : "=l"(r)
        : "l"(a), "l"(b));
    return r;
}

// a - b for canonical a, b: on a borrow, a - b + 2^64 - EPS = a - b + q
__device__ __forceinline__ uint64_t sub(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("{\n\t.reg .u32 a0, a1, b0, b1, d0, d1, br, z;\n\t"
        "mov.u32 z, 0;\n\t"
        "mov.b64 {a0, a1}, %1;\n\t"
        "mov.b64 {b0, b1}, %2;\n\t"
        "sub.cc.u32 d0, a0, b0;\n\t"
        "subc.cc.u32 d1, a1, b1;\n\t"
        "subc.u32 br, z, z;\n\t"      // 0, or 0xFFFFFFFF = EPS after a borrow
        "sub.cc.u32 d0, d0, br;\n\t"
        "subc.u32 d1, d1, z;\n\t"
        "mov.b64 %0, {d0, d1};\n\t}"
        : "=l"(r)
        : "l"(a), "l"(b));
    return r;
}

__device__ __forceinline__ uint64_t neg(uint64_t a) { return a ? Q - a : 0ull; }

// (hi * 2^64 + lo) mod q with hi = h1 * 2^32 + h0:  lo - h1 + h0 * (2^32 - 1), canonical.
// t = lo - h1 (minus EPS on a borrow: no second borrow since h1 < 2^32), u = h0 2^32 - h0,
// r = t + u with the same carry / canonical step as add (r + EPS when t + u or r + EPS carries).
__device__ __forceinline__ uint64_t reduce128(uint64_t lo, uint64_t hi) {
    uint64_t r;
    asm("{\n\t.reg .u32 l0, l1, h0, h1, t0, t1, u0, u1, r0, r1, s0, s1, br, c, z;\n\t.reg .pred p;\n\t"
        "mov.u32 z, 0;\n\t"
        "mov.b64 {l0, l1}, %1;\n\t"
        "mov.b64 {h0, h1}, %2;\n\t"
        "sub.cc.u32 t0, l0, h1;\n\t"
        "subc.cc.u32 t1, l1, z;\n\t"
        "subc.u32 br, z, z;\n\t"
        "sub.cc.u32 t0, t0, br;\n\t"
        "subc.u32 t1, t1, z;\n\t"
        "sub.cc.u32 u0, z, h0;\n\t"
        "subc.u32 u1, h0, z;\n\t"
        "add.cc.u32 r0, t0, u0;\n\t"
        "addc.cc.u32 r1, t1, u1;\n\t"
        "addc.u32 c, z, z;\n\t"
        "add.cc.u32 s0, r0, 0xFFFFFFFF;\n\t"
        "addc.cc.u32 s1, r1, z;\n\t"
        "addc.u32 c, c, z;\n\t"
        "setp.ne.u32 p, c, 0;\n\t"
        "selp.b32 r0, s0, r0, p;\n\t"
        "selp.b32 r1, s1, r1, p;\n\t"
        "mov.b64 %0, {r0, r1};\n\t}"
        : "=l"(r)
        : "l"(lo), "l"(hi));
    return r;
}

// a * b mod q, the 128-bit product from 32-bit multiply-adds
__device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b) {
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
    const uint32_t b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    uint32_t r0, r1, r2, r3;
    asm("mul.lo.u32 %0, %4, %6;\n\t"
        "mul.hi.u32 %1, %4, %6;\n\t"
        "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
        "madc.hi.u32 %2, %4, %7, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "madc.hi.u32 %3, %5, %7, 0;\n\t"
        "mad.lo.cc.u32 %2, %5, %7, %2;\n\t"
        "addc.u32 %3, %3, 0;"
        : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
        : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
    const uint64_t lo = ((uint64_t)r1 << 32) | r0;
    const uint64_t hi = ((uint64_t)r3 << 32) | r2;
    return reduce128(lo, hi);
}

// x * 2^S mod q for a compile-time shift S (any integer; 2^192 == 1, 2^96 == -1)
template <int S>
__device__ __forceinline__ uint64_t mul2k(uint64_t x) {
    constexpr int s = ((S % 192) + 192) % 192;
    if constexpr (s == 0) {
        return x;
    } else if constexpr (s >= 96) {
        return neg(mul2k<s - 96>(x));
    } else if constexpr (s >= 64) {
        return mul2k<s - 32>(mul2k<32>(x));
    } else {
        return reduce128(x << s, x >> (64 - s));
    }
}

// x * w^e for the primitive R-th root w_R = 2^(156 * 16 / R) (R | 16), conjugate (w^-e) if INV
template <int R, int E, bool INV>
__device__ __forceinline__ uint64_t rotr(uint64_t x) {
    constexpr int step = 156 * (16 / R);
    constexpr int e = ((E % R) + R) % R;
    return mul2k<(INV ? -step * e : step * e)>(x);
}

// In-register DFT of R points over GF(q), natural order in and out:
//   X_k = sum_n x_n w_R^{+-nk}   (w_R for the forward transform, w_R^-1 for INV; unscaled).
template <int R, bool INV>
struct NDft;

template <bool INV>
struct NDft<1, INV> {
    __device__ __forceinline__ static void run(uint64_t*) {}
};

template <bool INV>
struct NDft<2, INV> {
    __device__ __forceinline__ static void run(uint64_t* v) {
        const uint64_t a = v[0], b = v[1];
        v[0] = add(a, b);
        v[1] = sub(a, b);
    }
};

template <bool INV>
struct NDft<4, INV> {
    __device__ __forceinline__ static void run(uint64_t* v) {
        const uint64_t a0 = add(v[0], v[2]), a1 = sub(v[0], v[2]);
        const uint64_t b0 = add(v[1], v[3]);
        const uint64_t b1 = rotr<4, 1, INV>(sub(v[1], v[3]));
        v[0] = add(a0, b0);
        v[2] = sub(a0, b0);
        v[1] = add(a1, b1);
        v[3] = sub(a1, b1);
    }
};

// R = R1 * R2, decimation in frequency on the register array (as the FP64 DftSplit)
template <int R1, int R2, bool INV>
struct NDftSplit {
    static constexpr int R = R1 * R2;
    template <int N2, int K1>
    __device__ __forceinline__ static void twiddle_all(uint64_t (&a)[R1][R2]) {
        if constexpr (N2 < R2) {
            if constexpr (K1 < R1) {
                a[K1][N2] = rotr<R, N2 * K1, INV>(a[K1][N2]);
                twiddle_all<N2, K1 + 1>(a);
            } else {
                twiddle_all<N2 + 1, 0>(a);
            }
        }
    }
    __device__ __forceinline__ static void run(uint64_t* v) {
        uint64_t a[R1][R2];
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) {
            uint64_t col[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; ++n1) col[n1] = v[n1 * R2 + n2];
            NDft<R1, INV>::run(col);
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) a[k1][n2] = col[k1];
        }
        twiddle_all<0, 0>(a);
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) {
            NDft<R2, INV>::run(a[k1]);
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = a[k1][k2];
        }
    }
};

template <bool INV>
struct NDft<8, INV> {
    __device__ __forceinline__ static void run(uint64_t* v) { NDftSplit<2, 4, INV>::run(v); }
};
template <bool INV>
struct NDft<16, INV> {
    __device__ __forceinline__ static void run(uint64_t* v) { NDftSplit<4, 4, INV>::run(v); }
};

// Half table of the L-point transform, stored padded (entry r at qpad8(r) = r + r/16: strided
// pass indices spread over the 8-byte banks): t[qpad8(r)] = w_L^r, r < L/2. w_L^x for x < L is
// t[x] or, past L/2, -t[x - L/2] (w_L^(L/2) = -1): a read and a negation, no further product.
__host__ __device__ constexpr uint32_t qpad8(uint32_t r) { return r + (r >> 4); }
__host__ __device__ constexpr uint32_t qpad8_len(uint32_t qm) { return qm + (qm >> 4) + 1; }

template <int LOG_L>
__device__ __forceinline__ uint64_t twiddle(const uint64_t* __restrict__ t, uint32_t x, bool inv) {
    constexpr uint32_t L = 1u << LOG_L, HL = L / 2;
    if (inv) x = (L - x) & (L - 1);  // w^-x = w^(L - x)
    const uint64_t w = t[qpad8(x & (HL - 1))];
    return (x & HL) ? neg(w) : w;
}

}  // namespace gl
}  // namespace llg

#include "llg_fft.cuh"

namespace llg {
namespace gl {

// Radix pass S of the L-point NTT on the register array (same geometry, positions and exchange
// pattern as the FP64 passes of llg_fft.cuh; 8-byte field elements in the exchange buffer).
template <class G, int S, bool INV, bool SYNC_BEFORE_STORE, class SYNC>
__device__ __forceinline__ void radix_pass(uint64_t (&v)[G::E], uint64_t* __restrict__ buf,
                                           const uint64_t* __restrict__ qtw, int t, const SYNC& sync) {
    constexpr int R = G::radix(S);
    constexpr int L = G::len(S);
    constexpr int ST = G::stride(S);
    constexpr int B = G::E / R;
    constexpr bool LOAD = INV ? (S < G::P - 1) : (S > 0);
    constexpr bool STORE = INV ? (S > 0) : (S < G::P - 1);
#pragma unroll
    for (int h = 0; h < B; ++h) {
        const int beta = t * B + h;
        const int g = beta / ST, n2 = beta % ST;
        const int base = g * L + n2;
        uint64_t* vv = v + h * R;
        if constexpr (LOAD) {
#pragma unroll
            for (int n1 = 0; n1 < R; ++n1) vv[n1] = buf[phys(base + n1 * ST)];
        }
        if constexpr (!INV) {
            NDft<R, false>::run(vv);
            if constexpr (ST > 1) {
#pragma unroll
                for (int k1 = 1; k1 < R; ++k1)
                    vv[k1] = mul(vv[k1], twiddle<G::LOG_M_>(qtw, (uint32_t)(n2 * k1) << (G::LE * S), false));
            }
        } else {
            if constexpr (ST > 1) {
#pragma unroll
                for (int k1 = 1; k1 < R; ++k1)
                    vv[k1] = mul(vv[k1], twiddle<G::LOG_M_>(qtw, (uint32_t)(n2 * k1) << (G::LE * S), true));
            }
            NDft<R, true>::run(vv);
        }
        if constexpr (STORE && !SYNC_BEFORE_STORE) {
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) buf[phys(base + k1 * ST)] = vv[k1];
        }
    }
    if constexpr (STORE && SYNC_BEFORE_STORE) {
        sync();
#pragma unroll
        for (int h = 0; h < B; ++h) {
            const int beta = t * B + h;
            const int g = beta / ST, n2 = beta % ST;
            const int base = g * L + n2;
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) buf[phys(base + k1 * ST)] = v[h * R + k1];
        }
    }
}

template <class G, int S, class SYNC = CtaSync>
__device__ __forceinline__ void forward_from(uint64_t (&v)[G::E], uint64_t* buf, const uint64_t* qtw,
                                             int t, const SYNC& sync = SYNC()) {
    if constexpr (S < G::P) {
        radix_pass<G, S, false, false>(v, buf, qtw, t, sync);
        if constexpr (S < G::P - 1) sync();
        forward_from<G, S + 1, SYNC>(v, buf, qtw, t, sync);
    }
}

template <class G, int S, bool FIRST_SYNC = true, class SYNC = CtaSync>
__device__ __forceinline__ void inverse_from(uint64_t (&v)[G::E], uint64_t* buf, const uint64_t* qtw,
                                             int t, const SYNC& sync = SYNC()) {
    if constexpr (S >= 0) {
        radix_pass<G, S, true, FIRST_SYNC && S == G::P - 1>(v, buf, qtw, t, sync);
        if constexpr (S > 0) sync();
        inverse_from<G, S - 1, false, SYNC>(v, buf, qtw, t, sync);
    }
}

__device__ __forceinline__ uint64_t pow(uint64_t b, uint64_t e) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = mul(r, b);
        b = mul(b, b);
        e >>= 1;
    }
    return r;
}

// signed value of a canonical field element that holds an integer of magnitude < q/2
__device__ __forceinline__ long long lift(uint64_t z) {
    return (z > (Q >> 1)) ? -(long long)(Q - z) : (long long)z;
}
__device__ __forceinline__ uint64_t from_int(long long x) {
    return (x < 0) ? Q - (uint64_t)(-x) : (uint64_t)x;
}

}  // namespace gl
}  // namespace llg
