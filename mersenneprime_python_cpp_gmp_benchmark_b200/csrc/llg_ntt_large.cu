// Two-pass exact IBDWT over GF(2^64 - 2^32 + 1) for N = 2^14 .. 2^23, the residue resident in HBM
// as N field elements (8N bytes, the same footprint as the FP64 engine's N/2 complex values).
//
// Same four-step structure and carry scheme as the FP64 two-pass engine (llg_large.cu), with one
// digit per element instead of two (no real-FFT packing, so the column pass needs no partner
// column: one block per column, pointwise square):
//   row pass (kNttRowG consecutive rows a, all C columns):  inverse C-point NTT, unweight (and
//       1/N), signed lift, carry, "- 2", weight, forward C-point NTT;
//   column pass (one column c):  twiddle w_N^{ac}, forward R-point NTT, square, inverse, w_N^{-ac}.
// Carry: digit j = a + R b, so the chain runs down the rows of each column. Each row's carry-out
// is taken from zero (independent of its carry-in); the carry-in is absorbed with two
// renormalisations (hops 2, 3) whose own carries move one row further down, and the last, tiny
// remainder is added without renormalising (hop 4). A block's last row therefore publishes three
// carries, all computable without the previous block (a block has >= 3 rows); block k+1 reads them
// after a bounded wait on block k's flag (tickets in launch order keep block k resident). Block 0
// recomputes rows R-3 .. R-1 for the wrap-around carry into row 0 (2^p == 1).
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "llg_device.cuh"
#include "llg_fft.cuh"
#include "llg_internal.h"
#include "llg_ntt.cuh"

namespace llg {

namespace {

constexpr int kNttRowG = 4;
constexpr unsigned long long kNttSpinLimit = 1ull << 22;

__device__ __forceinline__ uint64_t twiddle_N(const NttLargeArgs& A, uint32_t x) {
    return gl::mul(__ldg(A.tw1 + (x & ((1u << A.tw_shift) - 1u))), __ldg(A.tw2 + (x >> A.tw_shift)));
}

}  // namespace

template <int LOG_C, int MODE>
__global__ void __launch_bounds__(kNttRowG * (1 << LOG_C) / 16, 2) ntt_row(const NttLargeArgs A) {
    using GC = SmallG<LOG_C>;
    constexpr int C = GC::M, TR = GC::T, E = GC::E, G = kNttRowG, T = G * TR;
    constexpr int RS = GC::PAD + 1;  // odd row stride (8-byte slots): the G rows of a slot hit G banks
    constexpr int QL = (int)gl::qpad8_len(C / 2);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* bufs = reinterpret_cast<uint64_t*>(smem_raw);   // G exchange buffers
    uint64_t* qtw = bufs + G * RS;                             // padded half table
    int* carr2 = reinterpret_cast<int*>(qtw + QL + (QL & 1));  // G x C hop-2 carry-outs
    int* carr3 = carr2 + G * C;                                // G x C hop-3 carry-outs
    long long* carr1 = reinterpret_cast<long long*>(bufs);     // G x C hop-1 carry-outs (reuses bufs)
    __shared__ int s_blk;
    __shared__ unsigned s_epoch;

    const int t = threadIdx.x, rg = t / TR, tr = t % TR;
    uint64_t* buf = bufs + rg * RS;
    const int N = 1 << A.logN, R = A.R;
    using RowSync = typename std::conditional<(TR >= 32), NamedSync, CtaSync>::type;
    RowSync gsync;
    if constexpr (TR >= 32) gsync = NamedSync{1u + (unsigned)rg, (unsigned)TR};

    if (t == 0) {
        const unsigned ep = *reinterpret_cast<volatile unsigned*>(&A.ctl->epoch);
        s_epoch = ep;
        if (MODE == LARGE_INIT) {
            s_blk = blockIdx.x;
        } else {
            const int b = (int)atomicAdd(&A.ctl->ticket[ep & 1], 1u);
            if (b == A.nblocks - 1) {
                // every block of this launch holds its ticket: both counters can be reset
                A.ctl->ticket[(ep + 1) & 1] = 0u;
                A.ctl->ticket[ep & 1] = 0u;
            }
            s_blk = b;
        }
    }
    for (int k = t; k < QL; k += T) qtw[k] = A.qtwC[k];
    __syncthreads();
    const int blk = s_blk;
    const unsigned ep = s_epoch;
    const int a0 = blk * G;
    const int a = a0 + rg;
    const int sA = __ldg(A.sA + a);

    uint64_t v[E];
    long long x[E];

    // unweight (with 1/N), lift, hop 1 of row `row` from the inverse transform in v
    auto hop1 = [&](int row, long long* c1out) {
        const int sa = __ldg(A.sA + row);
        const uint64_t iwa = __ldg(A.iwA + row);
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int b = tr + TR * i;
            const int sb = __ldg(A.sB + b);
            const bool o = sa + sb >= N;
            const int s = o ? sa + sb - N : sa + sb;
            uint64_t z = gl::mul(v[i], gl::mul(iwa, __ldg(A.iwB + b)));
            if (o) z = gl::add(z, z);  // w^-(s_j) = w^-sA w^-sB w^N, w^N = 2
            long long c;
            x[i] = balance(gl::lift(z), A.q + (s < A.rem), c);
            c1out[i] = c;
        }
    };
    auto bits_of = [&](int row, int b) {
        const int sa = __ldg(A.sA + row), sb = __ldg(A.sB + b);
        const int s = (sa + sb >= N) ? sa + sb - N : sa + sb;
        return A.q + (s < A.rem);
    };

    if constexpr (MODE == LARGE_INIT) {
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int b = tr + TR * i;
            x[i] = A.digits[(size_t)a + (size_t)R * b];
        }
    } else {
        // ---- block 0: wrap-around carries from rows R-3 .. R-1 (into row 0, column b + 1), the
        //      three rows transformed side by side (row group 3 repeats row R-1) ----
        if (blk == 0) {
            long long* hin1 = A.halo;  // c1 of row R-1, shifted to the column it feeds
            int* hin2 = reinterpret_cast<int*>(A.halo + C);
            int* hin3 = hin2 + C;
            const int ah = R - 3 + (rg < 3 ? rg : 2);
#pragma unroll
            for (int j = 0; j < E; ++j) v[j] = A.V[(size_t)(tr * E + j) * R + ah];
            gl::inverse_from<GC, GC::P - 1, false>(v, buf, qtw, tr, gsync);
            __syncthreads();  // the exchange buffers become the hop-1 carry array
            if (t == 0) {
                // rows R-3 .. R-1 are read: the last block may overwrite them
                __threadfence();
                *reinterpret_cast<volatile unsigned*>(&A.ctl->halo_read) = ep + 1u;
            }
            long long c1[E];
            hop1(ah, c1);
#pragma unroll
            for (int i = 0; i < E; ++i) carr1[rg * C + tr + TR * i] = c1[i];
            __syncthreads();
            if (rg == 1) {  // row R-2: hop 2 with row R-3's carry
#pragma unroll
                for (int i = 0; i < E; ++i) {
                    const int b = tr + TR * i;
                    long long c;
                    balance(x[i] + carr1[b], bits_of(ah, b), c);
                    carr2[b] = (int)c;
                }
            }
            __syncthreads();
            if (rg == 2) {  // row R-1: hops 2 and 3
#pragma unroll
                for (int i = 0; i < E; ++i) {
                    const int b = tr + TR * i;
                    const int nb = bits_of(ah, b);
                    long long c;
                    const long long y = balance(x[i] + carr1[C + b], nb, c);
                    const long long c2 = c;
                    balance(y + carr2[b], nb, c);
                    const int to = (b + 1) & (C - 1);
                    hin1[to] = c1[i];
                    hin2[to] = (int)c2;
                    hin3[to] = (int)c;
                }
            }
            __syncthreads();
        }

        // ---- load the block's rows (coalesced: kNttRowG contiguous elements per column slot) ----
        {
            uint64_t tmp[G * C / T];
#pragma unroll
            for (int r = 0; r < G * C / T; ++r) {
                const int qq = t + T * r, pos = qq / G, ra = qq % G;
                tmp[r] = A.V[(size_t)pos * R + a0 + ra];
            }
#pragma unroll
            for (int r = 0; r < G * C / T; ++r) {
                const int qq = t + T * r, pos = qq / G, ra = qq % G;
                bufs[ra * RS + phys(pos)] = tmp[r];
            }
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < E; ++j) v[j] = buf[phys(tr * E + j)];
        gl::inverse_from<GC, GC::P - 1, false>(v, buf, qtw, tr, gsync);
        __syncthreads();  // the exchange buffers become the hop-1 carry array

        // hop 1, every row
        {
            long long c1[E];
            hop1(a, c1);
#pragma unroll
            for (int i = 0; i < E; ++i) {
                const int b = tr + TR * i;
                carr1[rg * C + b] = c1[i];
                if (rg == G - 1) A.c1[(size_t)blk * C + b] = c1[i];
            }
        }
        __syncthreads();
        // hop 2, rows fed from inside the block
        if (rg >= 1) {
#pragma unroll
            for (int i = 0; i < E; ++i) {
                const int b = tr + TR * i;
                long long c;
                x[i] = balance(x[i] + carr1[(rg - 1) * C + b], bits_of(a, b), c);
                carr2[rg * C + b] = (int)c;
                if (rg == G - 1) A.c2[(size_t)blk * C + b] = (int)c;
            }
        }
        __syncthreads();
        // hop 3, rows whose hop-2 input is already known
        if (rg >= 2) {
#pragma unroll
            for (int i = 0; i < E; ++i) {
                const int b = tr + TR * i;
                long long c;
                x[i] = balance(x[i] + carr2[(rg - 1) * C + b], bits_of(a, b), c);
                carr3[rg * C + b] = (int)c;
                if (rg == G - 1) A.c3[(size_t)blk * C + b] = (int)c;
            }
        }
        __threadfence();  // carry-out stores ordered before the flag
        __syncthreads();
        if (t == 0) {
            __threadfence();
            *reinterpret_cast<volatile unsigned*>(&A.flags[blk]) = ep + 1u;
            if (blk > 0) wait_flag(&A.flags[blk - 1], ep + 1u, A.ctl, kNttSpinLimit);
        }
        __syncthreads();
        const long long* hin1 = A.halo;
        const int* hin2 = reinterpret_cast<const int*>(A.halo + C);
        const int* hin3 = hin2 + C;
        // hop 2 of the block's first row (previous block, or the wrap, and the "- 2" at digit 0)
        if (rg == 0) {
#pragma unroll
            for (int i = 0; i < E; ++i) {
                const int b = tr + TR * i;
                long long cin = (blk > 0) ? __ldcg(A.c1 + (size_t)(blk - 1) * C + b) : hin1[b];
                if (a == 0 && b == 0) cin -= 2;
                long long c;
                x[i] = balance(x[i] + cin, bits_of(a, b), c);
                carr2[b] = (int)c;
            }
        }
        __syncthreads();
        // hop 3 of the first two rows
        if (rg <= 1) {
#pragma unroll
            for (int i = 0; i < E; ++i) {
                const int b = tr + TR * i;
                const int cin = (rg == 1) ? carr2[b] : (blk > 0) ? __ldcg(A.c2 + (size_t)(blk - 1) * C + b) : hin2[b];
                long long c;
                x[i] = balance(x[i] + cin, bits_of(a, b), c);
                carr3[rg * C + b] = (int)c;
            }
        }
        __syncthreads();
        // hop 4: the remainder of the row above, not renormalised
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int b = tr + TR * i;
            const int cin = (rg > 0) ? carr3[(rg - 1) * C + b] : (blk > 0) ? __ldcg(A.c3 + (size_t)(blk - 1) * C + b) : hin3[b];
            x[i] += cin;
        }
        if (MODE == LARGE_FINAL || A.dump) {
#pragma unroll
            for (int i = 0; i < E; ++i) {
                const int b = tr + TR * i;
                A.digits[(size_t)a + (size_t)R * b] = (int)x[i];
            }
        }
        if constexpr (MODE == LARGE_FINAL) return;
        __syncthreads();  // carry reads done before the exchange buffers are reused
    }

    // ---- weight, forward row NTT, store ----
    const uint64_t wa = __ldg(A.wA + a);
#pragma unroll
    for (int i = 0; i < E; ++i) {
        const int b = tr + TR * i;
        const bool o = sA + __ldg(A.sB + b) >= N;
        uint64_t w = gl::mul(wa, __ldg(A.wB + b));
        if (o) w = gl::mul2k<191>(w);  // / 2
        v[i] = gl::mul(gl::from_int(x[i]), w);
    }
    gl::forward_from<GC, 0>(v, buf, qtw, tr, gsync);
#pragma unroll
    for (int j = 0; j < E; ++j) buf[phys(tr * E + j)] = v[j];
    if (MODE == LARGE_ITER && blk == A.nblocks - 1 && t == 0) {
        // rows R-3 .. R-1 are block 0's wrap-around input: wait (bounded) until it has read them
        wait_flag(&A.ctl->halo_read, ep + 1u, A.ctl, kNttSpinLimit);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < G * C / T; ++r) {
        const int qq = t + T * r, pos = qq / G, ra = qq % G;
        A.V[(size_t)pos * R + a0 + ra] = bufs[ra * RS + phys(pos)];
    }
}

template <int LOG_R>
__global__ void __launch_bounds__((1 << LOG_R) / 16, (LOG_R >= 13 ? 2 : 3)) ntt_col(const NttLargeArgs A) {
    using GR = SmallG<LOG_R>;
    constexpr int R = GR::M, TC = GR::T, E = GR::E;
    constexpr int QL = (int)gl::qpad8_len(R / 2);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* buf = reinterpret_cast<uint64_t*>(smem_raw);
    uint64_t* qtw = buf + GR::PAD;
    uint64_t* ptab = qtw + QL;  // E forward, E inverse
    const int tc = threadIdx.x;
    const int c = blockIdx.x;
    const int N = 1 << A.logN;
    for (int k = tc; k < QL; k += TC) qtw[k] = A.qtwR[k];
    // four-step twiddle w_N^{a c}, a = tc + TC i: w_N^{c tc} * w_N^{c TC i}
    for (int i = tc; i < E; i += TC) {
        const uint32_t xi = (uint32_t)(((uint64_t)c * TC * i) & (uint64_t)(N - 1));
        ptab[i] = twiddle_N(A, xi);
        ptab[E + i] = twiddle_N(A, (uint32_t)((N - xi) & (N - 1)));
    }
    const uint32_t xq = (uint32_t)(((uint64_t)c * tc) & (uint64_t)(N - 1));
    uint64_t* col = A.V + (size_t)__ldg(A.pos_of_c + c) * R;
    uint64_t v[E];
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = col[tc + TC * i];
    __syncthreads();
    {
        const uint64_t q = twiddle_N(A, xq);
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = gl::mul(v[i], gl::mul(q, ptab[i]));
    }
    gl::forward_from<GR, 0>(v, buf, qtw, tc);
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = gl::mul(v[j], v[j]);
    gl::inverse_from<GR, GR::P - 1, false>(v, buf, qtw, tc);
    {
        const uint64_t qi = twiddle_N(A, (uint32_t)((N - xq) & (N - 1)));
#pragma unroll
        for (int i = 0; i < E; ++i) col[tc + TC * i] = gl::mul(v[i], gl::mul(qi, ptab[E + i]));
    }
    if (c == 0 && tc == 0) atomicAdd(&A.ctl->epoch, 1u);
}

template <int LOG_C>
static size_t ntt_row_smem() {
    using GC = SmallGeom<LOG_C>;
    const size_t ql = gl::qpad8_len(GC::M / 2);
    return sizeof(uint64_t) * (kNttRowG * (GC::PAD + 1) + ql + (ql & 1)) + 2 * sizeof(int) * kNttRowG * GC::M;
}

template <int LOG_R>
static size_t ntt_col_smem() {
    using GR = SmallGeom<LOG_R>;
    return sizeof(uint64_t) * (GR::PAD + gl::qpad8_len(GR::M / 2) + 2 * GR::E);
}

template <int LOG_C, int MODE>
static cudaError_t ntt_row_attr() {
    return cudaFuncSetAttribute(ntt_row<LOG_C, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)ntt_row_smem<LOG_C>());
}

template <int LOG_C, int MODE>
static cudaError_t ntt_row_t(const NttLargeArgs& a, cudaStream_t st) {
    ntt_row<LOG_C, MODE><<<a.nblocks, kNttRowG * (1 << LOG_C) / 16, ntt_row_smem<LOG_C>(), st>>>(a);
    return cudaGetLastError();
}

template <int LOG_R>
static cudaError_t ntt_col_t(const NttLargeArgs& a, cudaStream_t st) {
    ntt_col<LOG_R><<<a.C, (1 << LOG_R) / 16, ntt_col_smem<LOG_R>(), st>>>(a);
    return cudaGetLastError();
}

template <int LOG_R>
static cudaError_t ntt_col_attr() {
    return cudaFuncSetAttribute(ntt_col<LOG_R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)ntt_col_smem<LOG_R>());
}

template <int LOG_C>
static cudaError_t ntt_row_attrs() {
    cudaError_t e = ntt_row_attr<LOG_C, LARGE_INIT>();
    if (!e) e = ntt_row_attr<LOG_C, LARGE_ITER>();
    if (!e) e = ntt_row_attr<LOG_C, LARGE_FINAL>();
    return e;
}

cudaError_t configure_ntt_large(int log_c, int log_r) {
    cudaError_t e;
    switch (log_c) {
        case 7: e = ntt_row_attrs<7>(); break;
        case 8: e = ntt_row_attrs<8>(); break;
        case 9: e = ntt_row_attrs<9>(); break;
        case 10: e = ntt_row_attrs<10>(); break;
        default: return cudaErrorInvalidValue;
    }
    if (e) return e;
    switch (log_r) {
        case 7: return ntt_col_attr<7>();
        case 8: return ntt_col_attr<8>();
        case 9: return ntt_col_attr<9>();
        case 10: return ntt_col_attr<10>();
        case 11: return ntt_col_attr<11>();
        case 12: return ntt_col_attr<12>();
        case 13: return ntt_col_attr<13>();
        default: return cudaErrorInvalidValue;
    }
}

template <int MODE>
static cudaError_t ntt_row_mode(int log_c, const NttLargeArgs& a, cudaStream_t st) {
    switch (log_c) {
        case 7: return ntt_row_t<7, MODE>(a, st);
        case 8: return ntt_row_t<8, MODE>(a, st);
        case 9: return ntt_row_t<9, MODE>(a, st);
        case 10: return ntt_row_t<10, MODE>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_ntt_row(int log_c, int mode, const NttLargeArgs& a, cudaStream_t st) {
    switch (mode) {
        case LARGE_INIT: return ntt_row_mode<LARGE_INIT>(log_c, a, st);
        case LARGE_ITER: return ntt_row_mode<LARGE_ITER>(log_c, a, st);
        case LARGE_FINAL: return ntt_row_mode<LARGE_FINAL>(log_c, a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_ntt_col(int log_r, const NttLargeArgs& a, cudaStream_t st) {
    switch (log_r) {
        case 7: return ntt_col_t<7>(a, st);
        case 8: return ntt_col_t<8>(a, st);
        case 9: return ntt_col_t<9>(a, st);
        case 10: return ntt_col_t<10>(a, st);
        case 11: return ntt_col_t<11>(a, st);
        case 12: return ntt_col_t<12>(a, st);
        case 13: return ntt_col_t<13>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace llg
