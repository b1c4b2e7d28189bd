// Shared-memory-exchanged in-register FFT of L = 2^LOG_L complex points (radix-16 passes, the
// last one radix 2/4/8/16), used for the whole-test kernel (L = M = N/2) and for the row and
// column passes of the two-pass engine. A group of T = L/16 threads owns one transform; thread t
// holds 16 values. Forward = decimation in frequency: natural order in (thread t holds element
// t + T*i in v[i]), mixed-radix digit-reversed order out (thread t holds positions 16t + j in
// v[j]; freq_of_pos / pos_of_freq translate). Inverse = the same passes retraced, back to natural
// order, unscaled (x L). The exchange buffer is one array of L + L/16 complex (16-byte) slots;
// phys() pads one slot per 16, which keeps every pass's access pattern at the minimum of four
// shared-memory wavefronts per warp access (at most five).
#pragma once

#include <cstdint>

#include "llg_device.cuh"

namespace llg {

// Twiddle table of a geometry: e^{-2 pi i r / M} at slot qpad(r) for r < M/4 (TW_QUARTER: the
// other quadrants by rotation), r < M/2 (TW_HALF: the other half by negation), or r < M (TW_FULL:
// one table read, no fold); TW_QUARTER_S: the quarter table at slot qpad_s(r).
enum { TW_QUARTER = 0, TW_HALF = 1, TW_FULL = 2, TW_QUARTER_S = 3 };

// L = 2^LOG_M points, E = 2^LOG_E values per thread (radix-E passes, the last one RLAST).
template <int LOG_M, int LOG_E = 4>
struct SmallGeom {
    static constexpr int M = 1 << LOG_M;
    static constexpr int N = 2 * M;
    static constexpr int LE = LOG_E;
    static constexpr int E = 1 << LOG_E;                  // complex values per thread
    static constexpr int T = M / E;                       // threads per transform
    static constexpr int P = (LOG_M + LOG_E - 1) / LOG_E; // radix passes
    static constexpr int RLAST = (LOG_M % LOG_E == 0) ? E : (1 << (LOG_M % LOG_E));
    static constexpr int PAD = M + M / 16;                // padded exchange array length (slots)
    static constexpr int W = (T + 31) / 32;               // warps
    static __host__ __device__ constexpr int radix(int s) { return s == P - 1 ? RLAST : E; }
    static __host__ __device__ constexpr int len(int s) { return M >> (LOG_E * s); }
    static __host__ __device__ constexpr int stride(int s) { return len(s) / radix(s); }
};

__device__ __forceinline__ int phys(int x) { return x + (x >> 4); }
// Exchange-buffer padding of one slot per 2^PADLOG (phys is PADLOG = 4).
template <int PADLOG>
__device__ __forceinline__ int physp(int x) { return x + (x >> PADLOG); }

// Digit reversal of the first P-1 radix-E digits: freq_of_pos(pos) = freq_rev(pos / RLAST) +
// (pos % RLAST) * (M / RLAST). For pos = t E + j (RLAST divides E) the first term depends on t and
// j / RLAST only, and w_M^{(pos % RLAST) M / RLAST} is an RLAST-th root of unity: the real-FFT
// split's twiddle w_M^freq is one table value per j / RLAST times an exact rotation.
template <class G>
__device__ __forceinline__ int freq_rev(int rest) {
    int k = 0;
#pragma unroll
    for (int s = 0; s < G::P - 1; ++s) {
        k = (k << G::LE) | (rest & (G::E - 1));
        rest >>= G::LE;
    }
    return k;
}

// Frequency index k of DIF output position pos (mixed radix E,...,E,RLAST digit reversal).
template <class G>
__device__ __forceinline__ int freq_of_pos(int pos) {
    int klast = pos % G::RLAST;
    int rest = pos / G::RLAST;
    int k = 0;
#pragma unroll
    for (int s = 0; s < G::P - 1; ++s) {
        k = (k << G::LE) | (rest & (G::E - 1));
        rest >>= G::LE;
    }
    // rest digits were stored most-significant-first as k1^(0); the loop above reversed them
    return k + klast * (G::M / G::RLAST);
}

template <class G>
__device__ __forceinline__ int pos_of_freq(int k) {
    const int klast = k / (G::M / G::RLAST);
    int low = k % (G::M / G::RLAST);
    int rest = 0;
#pragma unroll
    for (int s = 0; s < G::P - 1; ++s) {
        rest = (rest << G::LE) | (low & (G::E - 1));
        low >>= G::LE;
    }
    return rest * G::RLAST + klast;
}

// Barrier for the threads of one transform: the whole block, or a named barrier covering only the
// transform's own warps (several independent transforms per block then do not wait on each other).
struct CtaSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
struct NamedSync {
    unsigned id, nthreads;  // id 1..15; nthreads a multiple of 32
    __device__ __forceinline__ void operator()() const {
        asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
    }
    // signal arrival without waiting (the producer side of a producer/consumer pair of warps)
    __device__ __forceinline__ void arrive() const {
        asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
    }
};

// Twiddle e^{-2 pi i x / M} (conjugated when inv) for geometry G, from its table.
template <class G>
__device__ __forceinline__ double2 twiddle_g(const double2* __restrict__ q, uint32_t x, bool inv) {
    if constexpr (G::TWM == TW_FULL) {
        const double2 w = q[qpad(x & (uint32_t)(G::M - 1))];
        return inv ? conj2(w) : w;
    } else if constexpr (G::TWM == TW_HALF) {
        constexpr uint32_t H = (uint32_t)G::M / 2;
        const double2 w = q[qpad(x & (H - 1))];
        const bool ng = (x & H) != 0;  // e^{-2 pi i (r + M/2) / M} = -e^{-2 pi i r / M}
        return make_double2(ng ? -w.x : w.x, (ng != inv) ? -w.y : w.y);
    } else if constexpr (G::TWM == TW_QUARTER_S) {
        return twiddle<G::LOG_M_, true>(q, x, inv);
    } else {
        return twiddle<G::LOG_M_>(q, x, inv);
    }
}

// vv[k1] *= w^{x k1} (conjugated when INV) for k1 = 1 .. R-1, w = e^{-2 pi i / M}, x = n2 2^(LE S).
// Every twiddle read from the table, or (G::TWF, R >= 8) only those of k1 = 1, 2, 3 and
// k1 = 4, 8, 12 (R = 16; 4 for R = 8), the others formed as one product w^{x (k1 mod 4)}
// w^{x (k1 - k1 mod 4)}: 6 (4) table reads instead of 15 (7), each product within about an ulp.
template <class G, int R, bool INV>
__device__ __forceinline__ void apply_twiddles(double2* vv, const double2* __restrict__ qtw, uint32_t x) {
    if constexpr (G::TWF && R >= 8) {
        double2 lo[4], hi[4];
#pragma unroll
        for (int k = 1; k < 4; ++k) lo[k] = twiddle_g<G>(qtw, x * (uint32_t)k, INV);
#pragma unroll
        for (int k = 1; k < R / 4; ++k) hi[k] = twiddle_g<G>(qtw, x * (uint32_t)(4 * k), INV);
#pragma unroll
        for (int k1 = 1; k1 < R; ++k1) {
            const int l = k1 & 3, h = k1 >> 2;
            const double2 w = h == 0 ? lo[l] : (l == 0 ? hi[h] : cmul(hi[h], lo[l]));
            vv[k1] = cmul(vv[k1], w);
        }
    } else {
#pragma unroll
        for (int k1 = 1; k1 < R; ++k1) vv[k1] = cmul(vv[k1], twiddle_g<G>(qtw, x * (uint32_t)k1, INV));
    }
}

// Forward (INV=false) or inverse radix pass S on the register array v (E values).
// Forward: load (S > 0), DFT, twiddle w_L^{n2 k1}, store (S < P-1).
// Inverse: load (S < P-1), conj twiddle, inverse DFT, store (S > 0).
// ES: element stride of the exchange buffer. Slot x of this transform is buf[physp<PADLOG>(x) * ES],
// so ES transforms can share one buffer interleaved (transform r at buf + r), as the row pass of
// the two-pass engine does with the rows of a tile.
template <class G, int S, bool INV, bool SYNC_BEFORE_STORE, class SYNC, int ES = 1, int PADLOG = 4>
__device__ __forceinline__ void radix_pass(double2 (&v)[G::E], double2* __restrict__ buf,
                                           const double2* __restrict__ qtw, int t, const SYNC& sync) {
    constexpr int R = G::radix(S);
    constexpr int L = G::len(S);
    constexpr int ST = G::stride(S);
    constexpr int B = G::E / R;
    constexpr bool LOAD = INV ? (S < G::P - 1) : (S > 0);
    constexpr bool STORE = INV ? (S > 0) : (S < G::P - 1);
    // physp(base + n1 ST) = physp(base) + n1 * DST whenever the R slots of a butterfly never cross a
    // padding boundary (every 2^PADLOG slots) out of step with base: ST a multiple of 2^PADLOG, or
    // the whole group (L slots, L-aligned) inside one padding block. The offsets are then
    // compile-time constants.
    constexpr int PB = 1 << PADLOG;
    constexpr bool AFFINE = (ST % PB == 0) || (L <= PB);
    constexpr int DST = (ST % PB == 0) ? ST + ST / PB : ST;
#pragma unroll
    for (int h = 0; h < B; ++h) {
        const int beta = t * B + h;
        const int g = beta / ST, n2 = beta % ST;
        const int base = g * L + n2;
        const int pbase = physp<PADLOG>(base);
        double2* vv = v + h * R;
        if constexpr (LOAD) {
#pragma unroll
            for (int n1 = 0; n1 < R; ++n1) {
                const int x = AFFINE ? pbase + n1 * DST : physp<PADLOG>(base + n1 * ST);
                vv[n1] = buf[x * ES];
            }
        }
        if constexpr (!INV) {
            Dft<R, false>::run(vv);
            if constexpr (ST > 1) apply_twiddles<G, R, false>(vv, qtw, (uint32_t)n2 << (G::LE * S));
        } else {
            if constexpr (ST > 1) apply_twiddles<G, R, true>(vv, qtw, (uint32_t)n2 << (G::LE * S));
            Dft<R, true>::run(vv);
        }
        if constexpr (STORE && !SYNC_BEFORE_STORE) {
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) {
                const int x = AFFINE ? pbase + k1 * DST : physp<PADLOG>(base + k1 * ST);
                buf[x * ES] = vv[k1];
            }
        }
    }
    if constexpr (STORE && SYNC_BEFORE_STORE) {
        sync();
#pragma unroll
        for (int h = 0; h < B; ++h) {
            const int beta = t * B + h;
            const int g = beta / ST, n2 = beta % ST;
            const int base = g * L + n2;
            const int pbase = physp<PADLOG>(base);
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) {
                const int x = AFFINE ? pbase + k1 * DST : physp<PADLOG>(base + k1 * ST);
                buf[x * ES] = v[h * R + k1];
            }
        }
    }
}

// Forward passes S .. P-1 (pass S loads from buf unless S == 0).
template <class G, int S, class SYNC = CtaSync, int ES = 1, int PADLOG = 4>
__device__ __forceinline__ void forward_from(double2 (&v)[G::E], double2* buf, const double2* qtw,
                                             int t, const SYNC& sync = SYNC()) {
    if constexpr (S < G::P) {
        radix_pass<G, S, false, false, SYNC, ES, PADLOG>(v, buf, qtw, t, sync);
        if constexpr (S < G::P - 1) sync();
        forward_from<G, S + 1, SYNC, ES, PADLOG>(v, buf, qtw, t, sync);
    }
}

// Inverse passes S down to 0, starting from registers. FIRST_SYNC: a barrier between the first
// pass's arithmetic and its stores (needed when other threads may still read the positions it
// overwrites, e.g. a partner read of the same buffer).
template <class G, int S, bool FIRST_SYNC = true, class SYNC = CtaSync, int ES = 1, int PADLOG = 4>
__device__ __forceinline__ void inverse_from(double2 (&v)[G::E], double2* buf, const double2* qtw,
                                             int t, const SYNC& sync = SYNC()) {
    if constexpr (S >= 0) {
        radix_pass<G, S, true, FIRST_SYNC && S == G::P - 1, SYNC, ES, PADLOG>(v, buf, qtw, t, sync);
        if constexpr (S > 0) sync();
        inverse_from<G, S - 1, false, SYNC, ES, PADLOG>(v, buf, qtw, t, sync);
    }
}

// TF: the radix passes form their twiddles from fewer table reads (apply_twiddles).
template <int LOG_M_T, int LOG_E = 4, int TW = TW_QUARTER, bool TF = false>
struct SmallG : SmallGeom<LOG_M_T, LOG_E> {
    static constexpr int LOG_M_ = LOG_M_T;
    static constexpr int TWM = TW;
    static constexpr bool TWF = TF;
};

// Length (16-byte slots) of the twiddle table a geometry reads.
template <class G>
__host__ __device__ constexpr uint32_t twiddle_table_len() {
    if (G::TWM == TW_QUARTER_S) return qpad_s_len((uint32_t)G::M >> 2);
    return qpad_len((uint32_t)G::M >> (G::TWM == TW_FULL ? 0 : G::TWM == TW_HALF ? 1 : 2));
}

}  // namespace llg
