// Shared-memory-exchanged in-register FFT of L = 2^LOG_L complex points (radix-16 passes, the
// last one radix 2/4/8/16), used for the whole-test kernel (L = M = N/2) and for the row and
// column passes of the two-pass engine. A group of T = L/16 threads owns one transform; thread t
// holds 16 values. Forward = decimation in frequency: natural order in (thread t holds element
// t + T*i in v[i]), mixed-radix digit-reversed order out (thread t holds positions 16t + j in
// v[j]; freq_of_pos / pos_of_freq translate). Inverse = the same passes retraced, back to natural
// order, unscaled (x L). The exchange buffer is two padded double arrays (re, im) of
// L + L/16 entries; phys() pads one slot per 16 so strided accesses spread over the banks.
#pragma once

#include <cstdint>

#include "llg_device.cuh"

namespace llg {

template <int LOG_M>
struct SmallGeom {
    static constexpr int M = 1 << LOG_M;
    static constexpr int N = 2 * M;
    static constexpr int E = 16;               // complex values per thread
    static constexpr int T = M / E;            // threads per test
    static constexpr int P = (LOG_M + 3) / 4;  // radix passes
    static constexpr int RLAST = (LOG_M % 4 == 0) ? 16 : (1 << (LOG_M % 4));
    static constexpr int PAD = M + M / 16;     // padded exchange array length (doubles)
    static constexpr int W = (T + 31) / 32;    // warps
    static __host__ __device__ constexpr int radix(int s) { return s == P - 1 ? RLAST : 16; }
    static __host__ __device__ constexpr int len(int s) { return M >> (4 * s); }
    static __host__ __device__ constexpr int stride(int s) { return len(s) / radix(s); }
};

__device__ __forceinline__ int phys(int x) { return x + (x >> 4); }

// Frequency index k of DIF output position pos (mixed radix 16,...,16,RLAST digit reversal).
template <class G>
__device__ __forceinline__ int freq_of_pos(int pos) {
    int klast = pos % G::RLAST;
    int rest = pos / G::RLAST;
    int k = 0;
#pragma unroll
    for (int s = 0; s < G::P - 1; ++s) {
        k = (k << 4) | (rest & 15);
        rest >>= 4;
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
        rest = (rest << 4) | (low & 15);
        low >>= 4;
    }
    return rest * G::RLAST + klast;
}

// Forward (INV=false) or inverse radix pass S on the register array v (E values).
// Forward: load (S > 0), DFT, twiddle w_L^{n2 k1}, store (S < P-1).
// Inverse: load (S < P-1), conj twiddle, inverse DFT, store (S > 0).
template <class G, int S, bool INV, bool SYNC_BEFORE_STORE = false>
__device__ __forceinline__ void radix_pass(double2 (&v)[G::E], double* __restrict__ sre,
                                           double* __restrict__ sim,
                                           const double2* __restrict__ qtw, int t) {
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
        double2* vv = v + h * R;
        if constexpr (LOAD) {
#pragma unroll
            for (int n1 = 0; n1 < R; ++n1) {
                const int x = phys(base + n1 * ST);
                vv[n1] = make_double2(sre[x], sim[x]);
            }
        }
        if constexpr (!INV) {
            Dft<R, false>::run(vv);
            if constexpr (ST > 1) {
#pragma unroll
                for (int k1 = 1; k1 < R; ++k1)
                    vv[k1] = cmul(vv[k1], twiddle<G::LOG_M_>(qtw, (uint32_t)(n2 * k1) << (4 * S), false));
            }
        } else {
            if constexpr (ST > 1) {
#pragma unroll
                for (int k1 = 1; k1 < R; ++k1)
                    vv[k1] = cmul(vv[k1], twiddle<G::LOG_M_>(qtw, (uint32_t)(n2 * k1) << (4 * S), true));
            }
            Dft<R, true>::run(vv);
        }
        if constexpr (STORE && !SYNC_BEFORE_STORE) {
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) {
                const int x = phys(base + k1 * ST);
                sre[x] = vv[k1].x;
                sim[x] = vv[k1].y;
            }
        }
    }
    if constexpr (STORE && SYNC_BEFORE_STORE) {
        __syncthreads();
#pragma unroll
        for (int h = 0; h < B; ++h) {
            const int beta = t * B + h;
            const int g = beta / ST, n2 = beta % ST;
            const int base = g * L + n2;
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) {
                const int x = phys(base + k1 * ST);
                sre[x] = v[h * R + k1].x;
                sim[x] = v[h * R + k1].y;
            }
        }
    }
}

template <class G, int S>
__device__ __forceinline__ void forward_from(double2 (&v)[G::E], double* sre, double* sim,
                                             const double2* qtw, int t) {
    if constexpr (S < G::P) {
        radix_pass<G, S, false>(v, sre, sim, qtw, t);
        if constexpr (S < G::P - 1) __syncthreads();
        forward_from<G, S + 1>(v, sre, sim, qtw, t);
    }
}

template <class G, int S>
__device__ __forceinline__ void inverse_from(double2 (&v)[G::E], double* sre, double* sim,
                                             const double2* qtw, int t) {
    if constexpr (S >= 0) {
        radix_pass<G, S, true, S == G::P - 1>(v, sre, sim, qtw, t);
        if constexpr (S > 0) __syncthreads();
        inverse_from<G, S - 1>(v, sre, sim, qtw, t);
    }
}

template <int LOG_M_T>
struct SmallG : SmallGeom<LOG_M_T> {
    static constexpr int LOG_M_ = LOG_M_T;
};

}  // namespace llg
