// Whole-test-on-chip FP64 IBDWT Lucas-Lehmer kernel for transform lengths N = 32 .. 8192.
//
// One thread block owns one exponent and runs all of its squarings without leaving the SM: the
// residue lives in registers between iterations and shared memory is only the exchange buffer of
// the radix passes. This replaces, for small p, the reference's per-test loop of
// lucaslehmer.cpp:281-311 (FFTW r2c -> square -> c2r -> unweight/round -> carry) and the
// single-block GPU loop of cuda/ll_ntt.cu:91-163, with a different transform:
//
//   * the N real weighted digits are packed as M = N/2 complex values u_m = y_2m + i y_2m+1 and
//     transformed by an M-point complex FFT (radix-16 passes, radix-8 for M = 512, in-register
//     DFTs, one shared-memory exchange per pass, no bit reversal);
//   * the real-FFT split and the pointwise square are one step on the pair (k, M-k):
//       U'_k = [(3A - B)(A + B) - w^k (A - B)^2] / 4,  A = U_k, B = conj(U_{M-k}), w = e^{-2 pi i/M}
//     which equals DFT_M(z_even + i z_odd) for the cyclic square z = y * y;
//   * the inverse FFT retraces the passes (decimation in time) back to natural order, where each
//     thread holds u_m for m = t + T*i: unweight, round (1.5*2^52 shifter), max round-off,
//     balanced carry and re-weighting happen in registers. The carry chain m -> m+1 crosses from
//     thread t to t+1 (warp shuffle, one shared-memory hop per warp boundary); a thread's carry-out
//     does not depend on its carry-in (the incoming carry is folded into the first digit and its
//     small overflow left in the second), so one exchange per iteration suffices and the digits
//     stay balanced to within a few units.
//
// Round-off guard: every iteration's max |x - round(x)| is reduced into the block barrier of the
// carry exchange; above `abort_err` the test stops with status LLG_ST_ROUNDOFF and the host redoes
// it at the next larger N.
#include <cuda_runtime.h>

#include <cstdint>

#include "llg_device.cuh"
#include "llg_fft.cuh"
#include "llg_internal.h"

namespace llg {

// log2 of the complex values per thread for M = 2^log_m: 8 (radix-8 passes, twice the warps)
// for M = 2^9, where that takes no more passes than 16 (8 x 8 x 8 against 16 x 16 x 2); 16 else
__host__ __device__ constexpr int small_log_e(int log_m) { return log_m == 9 ? 3 : 4; }
// twiddle-table layout: spread (qpad_s) from M = 2^10 up, where the radix-16 passes' strided
// reads and the real-FFT split's digit-reversed reads conflict most in the qpad layout
__host__ __device__ constexpr int small_tw_layout(int log_m) { return log_m >= 10 ? TW_QUARTER_S : TW_QUARTER; }
template <int LOG_M>
using SmallGeo = SmallG<LOG_M, small_log_e(LOG_M), small_tw_layout(LOG_M), true>;

bool small_fp64_spread_table(int log_n) { return small_tw_layout(log_n - 1) == TW_QUARTER_S; }
// blocks per SM the kernel is built for: 128 registers a thread at 16 values, ~85 at 8
__host__ __device__ constexpr int small_min_blocks(int t, int le) {
    return t < 32 ? 16 : (le >= 4 ? 512 : 768) / t > 16 ? 16 : (le >= 4 ? 512 : 768) / t;
}

template <int LOG_M>
__global__ void __launch_bounds__(SmallGeo<LOG_M>::T, small_min_blocks(SmallGeo<LOG_M>::T, small_log_e(LOG_M)))
    ll_small_fp64(const SmallJob* __restrict__ jobs, const double2* __restrict__ qtw_g,
                  int64_t* __restrict__ digits_out, SmallResult* __restrict__ results,
                  float* __restrict__ errlog, double abort_err) {
    using G = SmallGeo<LOG_M>;
    constexpr int M = G::M, N = G::N, E = G::E, T = G::T, W = G::W;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* buf = reinterpret_cast<double2*>(smem_raw);          // exchange buffer, PAD slots
    double2* qtw = buf + G::PAD;                                   // padded quarter-wave table
    constexpr int QL = (int)twiddle_table_len<G>();
    double* wB = reinterpret_cast<double*>(qtw + QL);
    double* iwB = wB + E;
    int* sB = reinterpret_cast<int*>(iwB + E);
    double* cbuf = reinterpret_cast<double*>(sB + E + (E & 1 ? 1 : 0) + 2);  // W * E
    unsigned long long* serr = reinterpret_cast<unsigned long long*>(cbuf + W * E);  // 2
    // slot of the partner U_{M-k} of this thread's position t E + j, [j][t]: fixed for the whole
    // test, read in the real-FFT split instead of two digit reversals a value
    unsigned short* pslot = reinterpret_cast<unsigned short*>(serr + 2);  // E * T

    const int t = threadIdx.x;  // blockDim.x == T (a partial warp when T < 32)
    constexpr bool active = true;
    unsigned long long t_start = 0;
    if (t == 0) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_start));
    const SmallJob job = jobs[blockIdx.x];
    const uint64_t p = job.p;
    const uint64_t iters = job.iters;
    const int q = (int)(p >> (LOG_M + 1));          // p / N
    const int rem = (int)(p & (uint64_t)(N - 1));   // p % N

    for (int k = t; k < QL; k += blockDim.x) qtw[k] = qtw_g[k];
    for (int i = t; i < E; i += T) {
        // digit j = 2m + e with m = t + T*i: s_j = (sA(t,e) + sB(i)) mod N
        const uint64_t s = (uint64_t)(N - (int)(((uint64_t)2 * T * i * p) & (uint64_t)(N - 1))) &
                           (uint64_t)(N - 1);
        sB[i] = (int)s;
        wB[i] = exp2((double)s / (double)N);
        iwB[i] = exp2(-(double)s / (double)N) / (4.0 * (double)M);
    }
    for (int i = t; i < 2; i += T) serr[i] = 0ull;
#pragma unroll
    for (int j = 0; j < E; ++j) {
        const int kp = (M - freq_of_pos<G>(t * E + j)) & (M - 1);
        pslot[j * T + t] = (unsigned short)phys(pos_of_freq<G>(kp));
    }
    __syncthreads();

    // per-thread weight halves for the even (e=0) and odd (e=1) digit of each u_m
    int sA0 = 0, sA1 = 0;
    double wA0 = 1, wA1 = 1, iwA0 = 1, iwA1 = 1;
    if (active) {
        sA0 = (int)((uint64_t)(N - (int)(((uint64_t)(2 * t) * p) & (uint64_t)(N - 1))) & (uint64_t)(N - 1));
        sA1 = (int)((uint64_t)(N - (int)(((uint64_t)(2 * t + 1) * p) & (uint64_t)(N - 1))) & (uint64_t)(N - 1));
        wA0 = exp2((double)sA0 / (double)N);
        wA1 = exp2((double)sA1 / (double)N);
        iwA0 = exp2(-(double)sA0 / (double)N);
        iwA1 = exp2(-(double)sA1 / (double)N);
    }

    // kind of the two digits of column i, fixed for the whole test, 4 bits per column: bit 0 / 1:
    // digit 2m / 2m+1 has q + 1 bits (s < p mod N); bit 2 / 3: s_A + s_B wrapped past N (weight
    // = table product / 2, inverse weight x 2)
    uint32_t kinds[(E + 7) / 8];
#pragma unroll
    for (int w = 0; w < (E + 7) / 8; ++w) kinds[w] = 0u;
#pragma unroll
    for (int i = 0; i < E; ++i) {
        const int sb = sB[i];
        const bool o0 = sA0 + sb >= N, o1 = sA1 + sb >= N;
        const int s0 = o0 ? sA0 + sb - N : sA0 + sb;
        const int s1 = o1 ? sA1 + sb - N : sA1 + sb;
        const uint32_t kd = (uint32_t)(s0 < rem) | ((uint32_t)(s1 < rem) << 1) | ((uint32_t)o0 << 2) | ((uint32_t)o1 << 3);
        kinds[i / 8] |= kd << (4 * (i % 8));
    }
    auto kind = [&](int i) { return kinds[i / 8] >> (4 * (i % 8)); };
    // made opaque before each use: the weights and digit sizes derived from the kinds are then
    // formed where used, not hoisted into registers held across the transforms
    auto refresh_kinds = [&]() {
#pragma unroll
        for (int w = 0; w < (E + 7) / 8; ++w) asm volatile("" : "+r"(kinds[w]));
    };

    double2 v[E];
    // s_0 = 4: digit 0 (thread 0, i = 0, even) has weight a_0 = 1
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = make_double2(0.0, 0.0);
    if (t == 0) v[0].x = 4.0;

    const int lane = t & 31, warp = t >> 5;
    const int lastlane = (warp == W - 1) ? ((T - 1) & 31) : 31;
    const unsigned wmask = (T >= 32) ? 0xffffffffu : ((1u << T) - 1u);
    double maxerr = 0.0;
    uint64_t it = 0;
    uint32_t status = LLG_ST_OK;
    int x0s[E], x1s[E];

    for (;;) {
        forward_from<G, 0>(v, buf, qtw, t);
        // pair (k, M-k): real-FFT split + square, result scaled by 4 (folded into iwB)
        if (active) {
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const int x = phys(t * E + j);
                buf[x] = v[j];
            }
        }
        __syncthreads();
        if (active) {
            // w^k of position t E + j: one table value per j / RLAST, times w_RLAST^(j % RLAST)
            constexpr int RL = G::RLAST, NB = E / RL;
            double2 wk[NB];
#pragma unroll
            for (int h = 0; h < NB; ++h) wk[h] = twiddle_g<G>(qtw, (uint32_t)freq_rev<G>(t * NB + h), false);
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const int x = pslot[j * T + t];
                const double2 A = v[j], Bc = conj2(buf[x]);  // conj(U_{M-k})
                const double2 s = cadd(A, Bc), d = csub(A, Bc);
                const double2 a3 = make_double2(3.0 * A.x - Bc.x, 3.0 * A.y - Bc.y);
                const double2 d2 = make_double2((d.x - d.y) * (d.x + d.y), 2.0 * d.x * d.y);
                v[j] = csub(cmul(a3, s), cmul(wk[j / RL], rot_k<RL, false>(d2, j % RL)));
            }
            // the first inverse pass stores only after a barrier (partners may still be reading)
            inverse_from<G, G::P - 1>(v, buf, qtw, t);
        }

        // unweight, round, error, local carry (even -> odd digit); the carry-out of column i goes
        // to thread t+1 (lane shuffle) or, at a warp boundary, through cbuf after the barrier
        double lerr = 0.0;
        refresh_kinds();
        if (active) {
#pragma unroll
            for (int i = 0; i < E; ++i) {
                const uint32_t kd = kind(i);
                const double iw = iwB[i];
                const double a = v[i].x * (iwA0 * iw) * ((kd & 4u) ? 2.0 : 1.0);
                const double b = v[i].y * (iwA1 * iw) * ((kd & 8u) ? 2.0 : 1.0);
                long long la, lb;
                const double ra = round_shift(a, la), rb = round_shift(b, lb);
                lerr = fmax(lerr, fmax(fabs(a - ra), fabs(b - rb)));
                const int b0 = q + (int)(kd & 1u), b1 = q + (int)((kd >> 1) & 1u);  // digit sizes
                double c;
                double x0 = dsplit_e(ra, b0, c);
                const double x1 = dsplit_e(rb + c, b1, c);
                const double cout = c;
                if (lane == lastlane) cbuf[warp * E + i] = cout;
                const double cin = __shfl_up_sync(wmask, cout, 1);
                if (lane != 0) {
                    x0 = dsplit_e(x0 + cin, b0, c);
                    x1s[i] = d2i_exact(x1 + c);
                } else {
                    x1s[i] = d2i_exact(x1);
                }
                x0s[i] = d2i_exact(x0);
            }
        }
        maxerr = fmax(maxerr, lerr);
        if (errlog) atomicMax(&serr[it & 1], (unsigned long long)__double_as_longlong(lerr));
        const int bad = __syncthreads_or(lerr > abort_err);
        if (errlog && t == 0) {
            errlog[it] = (float)__longlong_as_double((long long)serr[it & 1]);
            serr[(it + 1) & 1] = 0ull;
        }
        refresh_kinds();
        if (active && lane == 0) {
#pragma unroll
            for (int i = 0; i < E; ++i) {
                double cin = (warp > 0) ? cbuf[(warp - 1) * E + i]
                                        : cbuf[(W - 1) * E + ((i + E - 1) % E)];  // m-1 wraps at m=0
                if (t == 0 && i == 0) cin -= 2.0;  // the "- 2" of s^2 - 2
                double c;
                x0s[i] = d2i_exact(dsplit_e((double)x0s[i] + cin, q + (int)(kind(i) & 1u), c));
                x1s[i] += (int)c;
            }
        }
        ++it;
        if (bad) {
            status = LLG_ST_ROUNDOFF;
            break;
        }
        if (it >= iters) break;
        refresh_kinds();
        if (active) {
#pragma unroll
            for (int i = 0; i < E; ++i) {
                const uint32_t kd = kind(i);
                const double w = wB[i];
                v[i].x = i2d_shift(x0s[i]) * (wA0 * w) * ((kd & 4u) ? 0.5 : 1.0);
                v[i].y = i2d_shift(x1s[i]) * (wA1 * w) * ((kd & 8u) ? 0.5 : 1.0);
            }
        }
    }

    if (active && digits_out) {
        int64_t* out = digits_out + (size_t)blockIdx.x * N;
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int m = t + T * i;
            out[2 * m] = x0s[i];
            out[2 * m + 1] = x1s[i];
        }
    }
    // block max of the round-off (non-negative doubles order like their bit patterns)
    __syncthreads();
    if (t == 0) serr[0] = 0ull;
    __syncthreads();
    atomicMax(&serr[0], (unsigned long long)__double_as_longlong(maxerr));
    __syncthreads();
    if (t == 0) {
        SmallResult r;
        r.max_err = __longlong_as_double((long long)serr[0]);
        r.iters_done = it;
        r.status = status;
        unsigned long long t_end;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_end));
        r.ns = t_end - t_start;
        results[blockIdx.x] = r;
    }
}

// p < 256: s <- s^2 - 2 mod 2^p - 1 on four 64-bit limbs (schoolbook square, shift-and-add
// reduction as in lucaslehmer.cpp:42-48), one thread per exponent. Exact; used where digits of
// an FFT length would hold too few bits for a stable balanced carry.
__device__ __forceinline__ void word_reduce(uint64_t (&s)[4], const uint64_t (&w)[8], int p) {
    // lo = w mod 2^p, hi = w >> p, s = lo + hi (both < 2^p), then conditional subtract of M
    uint64_t lo[4], hi[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int bit = 64 * i;
        lo[i] = (bit + 64 <= p) ? w[i] : (bit < p ? (w[i] & ((1ull << (p - bit)) - 1ull)) : 0ull);
        // hi limb i = bits [p + 64 i, p + 64 i + 64)
        const int q = (p + bit) >> 6, r = (p + bit) & 63;
        const uint64_t a0 = q < 8 ? w[q] : 0ull, a1 = q + 1 < 8 ? w[q + 1] : 0ull;
        hi[i] = r ? ((a0 >> r) | (a1 << (64 - r))) : a0;
    }
    unsigned __int128 c = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        c += (unsigned __int128)lo[i] + hi[i];
        s[i] = (uint64_t)c;
        c >>= 64;
    }
    // s < 2^(p+1): fold bit p back (2^p == 1) until s < 2^p, then s == M -> 0
    for (int guard = 0; guard < 3; ++guard) {
        const int q = p >> 6, r = p & 63;
        const uint64_t top = (q < 4) ? (s[q] >> r) : 0ull;
        if (!top) break;
        if (q < 4) s[q] &= (r ? ((1ull << r) - 1ull) : 0ull);
        unsigned __int128 cc = top;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            cc += s[i];
            s[i] = (uint64_t)cc;
            cc >>= 64;
        }
    }
    bool all = true;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int bit = 64 * i;
        const uint64_t full = (bit + 64 <= p) ? ~0ull : (bit < p ? ((1ull << (p - bit)) - 1ull) : 0ull);
        all = all && (s[i] == full);
    }
    if (all)
#pragma unroll
        for (int i = 0; i < 4; ++i) s[i] = 0ull;
}

__global__ void ll_word(const SmallJob* __restrict__ jobs, int n, uint64_t* __restrict__ res) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = (int)jobs[i].p;
    const uint64_t iters = jobs[i].iters;
    uint64_t s[4] = {4ull, 0ull, 0ull, 0ull};
    if (p == 2) s[0] = 1ull;  // 4 mod 3
    for (uint64_t k = 0; k < iters; ++k) {
        uint64_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            unsigned __int128 c = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                c += (unsigned __int128)s[a] * s[b] + w[a + b];
                w[a + b] = (uint64_t)c;
                c >>= 64;
            }
            w[a + 4] = (uint64_t)c;
        }
        word_reduce(s, w, p);
        // s - 2 mod M
        if (s[0] >= 2 || s[1] || s[2] || s[3]) {
            unsigned __int128 b = 2;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint64_t x = s[j];
                s[j] = x - (uint64_t)b;
                b = (x < (uint64_t)b) ? 1 : 0;
            }
        } else {  // s in {0, 1}: s - 2 + M = M - (2 - s)
            const uint64_t v = s[0];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int bit = 64 * j;
                s[j] = (bit + 64 <= p) ? ~0ull : (bit < p ? ((1ull << (p - bit)) - 1ull) : 0ull);
            }
            s[0] -= 2ull - v;
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) res[(size_t)i * 4 + j] = s[j];
}

cudaError_t launch_word(const SmallJob* jobs, int njobs, uint64_t* res, cudaStream_t st) {
    ll_word<<<(njobs + 127) / 128, 128, 0, st>>>(jobs, njobs, res);
    return cudaGetLastError();
}

template <int LOG_M>
static size_t small_smem_bytes() {
    using G = SmallGeo<LOG_M>;
    size_t b = sizeof(double2) * G::PAD;
    b += sizeof(double2) * twiddle_table_len<G>();
    b += 2 * sizeof(double) * G::E + sizeof(int) * (G::E + (G::E & 1 ? 1 : 0) + 2);
    b += sizeof(double) * G::W * G::E + 2 * sizeof(unsigned long long);
    b += sizeof(unsigned short) * G::E * G::T;  // partner slots of the real-FFT split
    return b;
}

template <int LOG_M>
static cudaError_t launch_small_t(const SmallJob* jobs, int njobs, const double2* qtw,
                                  int64_t* digits, SmallResult* results, float* errlog,
                                  double abort_err, cudaStream_t st) {
    using G = SmallGeo<LOG_M>;
    const size_t smem = small_smem_bytes<LOG_M>();
    static PerDeviceOnce configured;
    if (!configured.done()) {
        cudaError_t e = cudaFuncSetAttribute(ll_small_fp64<LOG_M>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured.mark();
    }
    ll_small_fp64<LOG_M><<<njobs, G::T, smem, st>>>(jobs, qtw, digits, results, errlog, abort_err);
    return cudaGetLastError();
}

cudaError_t launch_small_fp64(int log_n, const SmallJob* jobs, int njobs, const double2* qtw,
                              int64_t* digits, SmallResult* results, float* errlog,
                              double abort_err, cudaStream_t st) {
    switch (log_n - 1) {
        case 4: return launch_small_t<4>(jobs, njobs, qtw, digits, results, errlog, abort_err, st);
        case 5: return launch_small_t<5>(jobs, njobs, qtw, digits, results, errlog, abort_err, st);
        case 6: return launch_small_t<6>(jobs, njobs, qtw, digits, results, errlog, abort_err, st);
        case 7: return launch_small_t<7>(jobs, njobs, qtw, digits, results, errlog, abort_err, st);
        case 8: return launch_small_t<8>(jobs, njobs, qtw, digits, results, errlog, abort_err, st);
        case 9: return launch_small_t<9>(jobs, njobs, qtw, digits, results, errlog, abort_err, st);
        case 10: return launch_small_t<10>(jobs, njobs, qtw, digits, results, errlog, abort_err, st);
        case 11: return launch_small_t<11>(jobs, njobs, qtw, digits, results, errlog, abort_err, st);
        case 12: return launch_small_t<12>(jobs, njobs, qtw, digits, results, errlog, abort_err, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace llg
