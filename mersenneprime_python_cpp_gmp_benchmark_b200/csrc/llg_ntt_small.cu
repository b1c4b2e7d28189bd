// Whole-test-on-chip exact IBDWT over GF(2^64 - 2^32 + 1) for N = 32 .. 8192 (the Goldilocks NTT
// engine). One block per exponent, all squarings on chip. The reference's kernel for this
// (cuda/ll_ntt.cu:74-167) runs radix-2 stages with a barrier per stage and a carry loop that
// repeats until no carry is left; here:
//   * radix-16 passes in registers (internal twiddles are powers of 2, i.e. shifts), one exchange
//     through shared memory per pass, no bit reversal (the pointwise square ignores order);
//   * weights w^s with w an N-th root of 2 in the field (s = ceil(jp/N) N - jp), computed per
//     thread once per test as w^sA * w^sB (digit m = t + T*i: sA from the thread, sB from i);
//   * the carry in four fixed hops: each digit's carry-out is taken from zero (independent of its
//     carry-in), the carry-in is absorbed with a renormalisation twice and the remainder (|r| < 2 in
//     practice) added to the next digit, so the result is exact and three exchanges suffice.
// Exactness: every convolution output is an integer below N 2^(2B-2) < q/2 for the lengths chosen
// by the host (B = bits of the largest digit), so the field value is the integer.
#include <cuda_runtime.h>

#include <cstdint>

#include "llg_device.cuh"
#include "llg_fft.cuh"
#include "llg_internal.h"
#include "llg_ntt.cuh"

namespace llg {

template <int LOG_N>
__global__ void __launch_bounds__(SmallGeom<LOG_N>::T)
    ll_small_ntt(const SmallJob* __restrict__ jobs, const uint64_t* __restrict__ qtw_g, NttConst K,
                 int64_t* __restrict__ digits_out, SmallResult* __restrict__ results) {
    using G = SmallG<LOG_N>;
    constexpr int N = G::M, E = G::E, T = G::T, W = G::W;
    constexpr int QL = (int)gl::qpad8_len(N / 2);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* buf = reinterpret_cast<uint64_t*>(smem_raw);  // exchange buffer, PAD slots
    uint64_t* qtw = buf + G::PAD;                            // padded half table
    uint64_t* wB = qtw + QL;                                 // E: w^sB(i)
    uint64_t* iwB = wB + E;                                  // E: w^-sB(i) / N
    long long* cbuf = reinterpret_cast<long long*>(iwB + E); // 3 hops x W x E carry slots
    int* sB = reinterpret_cast<int*>(cbuf + 3 * W * E);      // E

    const int t = threadIdx.x;
    unsigned long long t_start = 0;
    if (t == 0) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_start));
    const SmallJob job = jobs[blockIdx.x];
    const uint64_t p = job.p, iters = job.iters;
    const int qp = (int)(p >> LOG_N);
    const int rem = (int)(p & (uint64_t)(N - 1));

    for (int k = t; k < QL; k += T) qtw[k] = qtw_g[k];
    for (int i = t; i < E; i += T) {
        // digit m = t + T i: s_m = (sA(t) + sB(i)) mod N, sB(i) = (-T i p) mod N
        const int s = (int)((uint64_t)(N - (int)(((uint64_t)T * i * p) & (uint64_t)(N - 1))) & (uint64_t)(N - 1));
        sB[i] = s;
        wB[i] = gl::pow(K.root2, (uint64_t)s);
        iwB[i] = gl::mul(gl::pow(K.inv_root2, (uint64_t)s), K.invN);
    }
    const int sA = (int)((uint64_t)(N - (int)(((uint64_t)t * p) & (uint64_t)(N - 1))) & (uint64_t)(N - 1));
    const uint64_t wA = gl::pow(K.root2, (uint64_t)sA);
    const uint64_t iwA = gl::pow(K.inv_root2, (uint64_t)sA);
    __syncthreads();

    const int lane = t & 31, warp = t >> 5;
    const int lastlane = (warp == W - 1) ? ((T - 1) & 31) : 31;
    const unsigned wmask = (T >= 32) ? 0xffffffffu : ((1u << T) - 1u);

    uint64_t v[E];
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = 0ull;
    if (t == 0) v[0] = 4ull;  // s_0 = 4 at digit 0 (weight 1)
    long long x[E];
    uint64_t it = 0;

    // carry exchange of one hop: cin[i] = carry-out of element m - 1 (element m = t + T i)
    auto exchange = [&](long long (&c)[E], int hop) {
        long long* cb = cbuf + hop * W * E;
        if (lane == lastlane) {
#pragma unroll
            for (int i = 0; i < E; ++i) cb[warp * E + i] = c[i];
        }
        long long up[E];
#pragma unroll
        for (int i = 0; i < E; ++i) up[i] = __shfl_up_sync(wmask, c[i], 1);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < E; ++i) {
            if (lane != 0)
                c[i] = up[i];
            else
                c[i] = (warp > 0) ? cb[(warp - 1) * E + i] : cb[(W - 1) * E + ((i + E - 1) % E)];
        }
    };

    for (;;) {
        gl::forward_from<G, 0>(v, buf, qtw, t);
#pragma unroll
        for (int j = 0; j < E; ++j) v[j] = gl::mul(v[j], v[j]);
        gl::inverse_from<G, G::P - 1, false>(v, buf, qtw, t);
        // unweight (with 1/N), lift to signed, hop 1 from zero
        long long c[E];
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int sbi = sB[i];
            const bool o = sA + sbi >= N;
            const int s = o ? sA + sbi - N : sA + sbi;
            uint64_t z = gl::mul(v[i], gl::mul(iwA, iwB[i]));
            if (o) z = gl::add(z, z);  // w^-(s - N) ... : w^-s_m = w^-sA w^-sB w^N, w^N = 2
            long long cc;
            x[i] = balance(gl::lift(z), qp + (s < rem), cc);
            c[i] = cc;
        }
        exchange(c, 0);
        // hop 2: absorb the neighbour's carry (and the "- 2" at digit 0)
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int sbi = sB[i];
            const int s = (sA + sbi >= N) ? sA + sbi - N : sA + sbi;
            long long cin = c[i];
            if (t == 0 && i == 0) cin -= 2;
            long long cc;
            x[i] = balance(x[i] + cin, qp + (s < rem), cc);
            c[i] = cc;
        }
        exchange(c, 1);
        // hop 3: absorb the (small) second carry, renormalise once more
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int sbi = sB[i];
            const int s = (sA + sbi >= N) ? sA + sbi - N : sA + sbi;
            long long cc;
            x[i] = balance(x[i] + c[i], qp + (s < rem), cc);
            c[i] = cc;
        }
        exchange(c, 2);
        // hop 4: the remainder (|c| <= 1 in practice) stays in the digit
#pragma unroll
        for (int i = 0; i < E; ++i) x[i] += c[i];
        ++it;
        if (it >= iters) break;
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const bool o = sA + sB[i] >= N;
            uint64_t w = gl::mul(wA, wB[i]);
            if (o) w = gl::mul2k<191>(w);  // / 2 (2^-1 == 2^191)
            v[i] = gl::mul(gl::from_int(x[i]), w);
        }
    }

    if (digits_out) {
        int64_t* out = digits_out + (size_t)blockIdx.x * N;
#pragma unroll
        for (int i = 0; i < E; ++i) out[t + T * i] = x[i];
    }
    if (t == 0) {
        SmallResult r;
        r.max_err = 0.0;
        r.iters_done = it;
        r.status = LLG_ST_OK;
        unsigned long long t_end;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_end));
        r.ns = t_end - t_start;
        results[blockIdx.x] = r;
    }
}

template <int LOG_N>
static size_t small_ntt_smem() {
    using G = SmallGeom<LOG_N>;
    return sizeof(uint64_t) * (G::PAD + gl::qpad8_len(G::M / 2) + 2 * G::E) +
           sizeof(long long) * 3 * G::W * G::E + sizeof(int) * G::E;
}

template <int LOG_N>
static cudaError_t launch_small_ntt_t(const SmallJob* jobs, int njobs, const uint64_t* qtw, NttConst K,
                                      int64_t* digits, SmallResult* results, cudaStream_t st) {
    using G = SmallGeom<LOG_N>;
    const size_t smem = small_ntt_smem<LOG_N>();
    cudaError_t e = cudaFuncSetAttribute(ll_small_ntt<LOG_N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    ll_small_ntt<LOG_N><<<njobs, G::T, smem, st>>>(jobs, qtw, K, digits, results);
    return cudaGetLastError();
}

cudaError_t launch_small_ntt(int log_n, const SmallJob* jobs, int njobs, const uint64_t* qtw, NttConst K,
                             int64_t* digits, SmallResult* results, cudaStream_t st) {
    switch (log_n) {
        case 5: return launch_small_ntt_t<5>(jobs, njobs, qtw, K, digits, results, st);
        case 6: return launch_small_ntt_t<6>(jobs, njobs, qtw, K, digits, results, st);
        case 7: return launch_small_ntt_t<7>(jobs, njobs, qtw, K, digits, results, st);
        case 8: return launch_small_ntt_t<8>(jobs, njobs, qtw, K, digits, results, st);
        case 9: return launch_small_ntt_t<9>(jobs, njobs, qtw, K, digits, results, st);
        case 10: return launch_small_ntt_t<10>(jobs, njobs, qtw, K, digits, results, st);
        case 11: return launch_small_ntt_t<11>(jobs, njobs, qtw, K, digits, results, st);
        case 12: return launch_small_ntt_t<12>(jobs, njobs, qtw, K, digits, results, st);
        case 13: return launch_small_ntt_t<13>(jobs, njobs, qtw, K, digits, results, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace llg
