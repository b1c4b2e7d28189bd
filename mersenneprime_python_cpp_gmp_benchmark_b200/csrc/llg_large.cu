// Two-pass FP64 IBDWT squaring for N = 2^14 .. 2^23 with the residue resident in HBM.
//
// The M = N/2 packed complex values u_m (m = a + R*b: row a < R, column b < C, M = R*C) are
// transformed by the four-step method. One squaring is two kernels, i.e. two read+write sweeps of
// the 16*M-byte state -- the fewest a transform of this size allows when each pass's working set
// must fit on chip (the reference does one monolithic FFTW transform per direction,
// lucaslehmer.cpp:283,288, and an O(N) host loop for each of weight, unweight and carry,
// lucaslehmer.cpp:282,289-310):
//
//   row pass (one block = G consecutive rows, G = 2, 4 or 8, all C columns):
//       inverse C-point FFT                                   (end of the previous squaring)
//       unweight, round, max round-off, carry, "- 2"
//       weight, forward C-point FFT                           (start of this squaring)
//   column pass (one block = the column pair c, C-c):
//       twiddle w_M^{ac}, forward R-point FFT, real-FFT split + pointwise square over the pair
//       (k, M-k), inverse R-point FFT, twiddle w_M^{-ac}
//
// The state is stored column-slot-major (element (a, pos) at pos*R + a), so a row block reads
// and writes G contiguous complex values (16 G bytes) per column slot and a column block reads
// and writes its columns contiguously.
//
// Carry. Digits 2m, 2m+1 of row a carry into row a+1 (m -> m+1 is a -> a+1), so the chain runs
// down the rows of each column b. Each row's carry-out is computed from that row's rounded values
// alone (two-digit chain started at zero); the incoming carry is folded into the first digit and
// the small remainder into the second, which keeps every digit within a few units of balanced and
// makes carry-outs independent of carry-ins. Inside a block the carries pass through shared
// memory; between blocks block k publishes its last row's carry-outs and a flag, and block k+1
// reads them after a bounded wait. Only the block's first row waits for that flag (and its
// second row for the first row's result): the other rows finish their carries from inside the
// block and go on to the forward FFT meanwhile. Blocks take tickets in launch order, so the block waited on is
// always resident or finished. The wrap-around carry into row 0 (2^p == 1) comes from row R-1;
// block 0 runs the last block's rows through the same code first, instead of waiting on the last
// block, and the last block waits (bounded) until block 0 has read them before overwriting them.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "llg_device.cuh"
#include "llg_fft.cuh"
#include "llg_host.h"
#include "llg_internal.h"

namespace llg {

namespace {

constexpr unsigned long long kSpinLimit = 1ull << 22;  // x ~64 ns: ~0.3 s, then give up + flag

__device__ __forceinline__ double2 twiddle_M(const LargeArgs& A, uint32_t x, bool inv) {
    const double2 a = __ldg(A.tw1 + (x & ((1u << A.tw_shift) - 1u)));
    const double2 b = __ldg(A.tw2 + (x >> A.tw_shift));
    const double2 w = cmul(a, b);
    return inv ? conj2(w) : w;
}

}  // namespace

__host__ __device__ constexpr int large_row_threads(int log_c, int g) {
    return g * (1 << log_c) / (1 << large_row_log_e(log_c, g));
}
// blocks per SM the row kernel is built for: 128 registers a thread at 16 values, 64 at 8
__host__ __device__ constexpr int large_row_min_blocks(int log_c, int g) {
    const int t = large_row_threads(log_c, g) < 32 ? 32 : large_row_threads(log_c, g);
    const int b = (large_row_log_e(log_c, g) >= 4 ? 512 : 1024) / t;
    return b > 16 ? 16 : b;
}

template <int LOG_C, int G, int MODE>
__global__ void __launch_bounds__(large_row_threads(LOG_C, G), large_row_min_blocks(LOG_C, G))
    large_row(const LargeArgs A) {
    using GC = SmallG<LOG_C, large_row_log_e(LOG_C, G), TW_FULL>;  // full twiddle table
    constexpr int C = GC::M, TR = GC::T, E = GC::E, T = G * TR;
    static_assert(T % 32 == 0, "whole warps");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int RS = GC::PAD + 1;  // row-buffer stride: odd, so the rows of a slot hit different banks
    constexpr int QL = (int)twiddle_table_len<GC>();
    double2* bufs = reinterpret_cast<double2*>(smem_raw);  // G exchange buffers of RS slots
    double2* qtw = bufs + G * RS;                            // padded twiddle table (C-point)
    double* carr = reinterpret_cast<double*>(bufs);          // G x C hop-1 carry-outs (reuses bufs)
    double* carr2 = carr + G * C;                            // G x C hop-2 carry-outs
    double* late = reinterpret_cast<double*>(qtw + QL);     // C: row 0's hop-2 carry-outs, for row 1
    double* hin = reinterpret_cast<double*>(A.halo);         // C: wrap carry into row 0 (hop 2)
    double* hin2 = hin + C;                                  // C: wrap carry into row 0 (hop 3)
    __shared__ unsigned long long s_err;
    __shared__ int s_blk;
    __shared__ unsigned s_epoch;

    const int t = threadIdx.x, rg = t / TR, tr = t % TR;
    double2* buf = bufs + rg * RS;
    const int N = 1 << A.logN, R = A.R;
    // each row's FFT exchanges wait only on that row's warps (named barrier 1 + rg)
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
        s_err = 0ull;
    }
    __syncthreads();
    const int blk = s_blk;
    const unsigned ep = s_epoch;
    const int a0 = blk * G;
    const int a = a0 + rg;
    // digit sizes: b = q or q + 1 bits, as 2^b and 2^-b
    const double pw0 = pow2(A.q), pw1 = pow2(A.q + 1), iv0 = pow2(-A.q), iv1 = pow2(-A.q - 1);
    // column weight exponent sB(b) = (-2 R b p) mod N, from 32-bit products (N <= 2^23 < 2^32)
    const uint32_t kB = (uint32_t)(2 * R) * (uint32_t)A.rem;
    auto sB_of = [&](int b) { return (int)((0u - kB * (uint32_t)b) & (uint32_t)(N - 1)); };

    double2 v[E];
    double x0s[E], x1s[E];

    if constexpr (MODE == LARGE_INIT) {
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int b = tr + TR * i;
            const size_t m = (size_t)a + (size_t)R * b;
            const int2 d = *reinterpret_cast<const int2*>(A.digits + 2 * m);
            x0s[i] = (double)d.x;
            x1s[i] = (double)d.y;
        }
        for (int k = t; k < QL; k += T) qtw[k] = A.qtwC[k];
        __syncthreads();
    } else {
        double lerr = 0.0;
        // Phase 0 (block 0 only): the last block's rows R-G .. R-1 through the same inverse FFT
        // and hops 1-2, for the carry-outs of row R-1 that wrap into row 0 (2^p == 1), exactly as
        // the last block computes and publishes them. Phase 1: the block's own rows.
#pragma unroll 1
        for (int ph = (blk == 0) ? 0 : 1; ph < 2; ++ph) {
            const int base = ph ? a0 : R - G;
            const int ar = base + rg;
            // ---- load rows base .. base+G-1 (coalesced: G contiguous values per column slot) ----
            {
                double2 tmp[G * C / T];
#pragma unroll
                for (int r = 0; r < G * C / T; ++r) {
                    const int qq = t + T * r, pos = qq / G, ra = qq % G;
                    tmp[r] = A.V[(size_t)pos * R + base + ra];
                }
                // the twiddle table (L2-resident) is fetched while the rows' loads are in flight
                if (ph == 0 || blk != 0)
                    for (int k = t; k < QL; k += T) qtw[k] = A.qtwC[k];
#pragma unroll
                for (int r = 0; r < G * C / T; ++r) {
                    const int qq = t + T * r, pos = qq / G, ra = qq % G;
                    bufs[ra * RS + phys(pos)] = tmp[r];
                }
            }
            __syncthreads();
            if (ph == 0 && t == 0) {
                // rows R-G .. R-1 are read: the last block may overwrite them
                __threadfence();
                *reinterpret_cast<volatile unsigned*>(&A.ctl->halo_read) = ep + 1u;
            }
#pragma unroll
            for (int j = 0; j < E; ++j) v[j] = buf[phys(tr * E + j)];
            inverse_from<GC, GC::P - 1, false>(v, buf, qtw, tr, gsync);
            __syncthreads();  // the exchange buffers become the carry arrays

            // ---- hop 1: unweight, round, round-off, two-digit chain per (row, column) from zero;
            //      the carry-out goes to the next row. ----
            const int sA0 = __ldg(A.sA + 2 * ar), sA1 = __ldg(A.sA + 2 * ar + 1);
            const double ia0 = __ldg(A.iwA + 2 * ar), ia1 = __ldg(A.iwA + 2 * ar + 1);
#pragma unroll
            for (int i = 0; i < E; ++i) {
                const int b = tr + TR * i;
                const int sb = sB_of(b);
                const double iwb = __ldg(A.iwB + b);
                const bool o0 = sA0 + sb >= N, o1 = sA1 + sb >= N;
                const int s0 = o0 ? sA0 + sb - N : sA0 + sb, s1 = o1 ? sA1 + sb - N : sA1 + sb;
                const bool w0 = s0 < A.rem, w1 = s1 < A.rem;  // digit of q + 1 bits
                const double va = v[i].x * (ia0 * iwb) * (o0 ? 2.0 : 1.0);
                const double vb = v[i].y * (ia1 * iwb) * (o1 ? 2.0 : 1.0);
                long long ia, ib;
                const double ra = round_shift(va, ia), rb = round_shift(vb, ib);
                lerr = fmax(lerr, fmax(fabs(va - ra), fabs(vb - rb)));
                double c;
                x0s[i] = dsplit(ra, w0 ? iv1 : iv0, w0 ? pw1 : pw0, c);
                x1s[i] = dsplit(rb + c, w1 ? iv1 : iv0, w1 ? pw1 : pw0, c);
                carr[rg * C + b] = c;
            }
            // the block's round-off max: one shared atomic per warp
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) lerr = fmax(lerr, __shfl_xor_sync(0xffffffffu, lerr, o));
            if ((t & 31) == 0) atomicMax(&s_err, (unsigned long long)__double_as_longlong(lerr));
            __syncthreads();
            // ---- hop 2 for rows fed from inside the block ----
            if (rg > 0) {
#pragma unroll
                for (int i = 0; i < E; ++i) {
                    const int b = tr + TR * i;
                    const int sb = sB_of(b);
                    const bool o0 = sA0 + sb >= N, o1 = sA1 + sb >= N;
                    const int s0 = o0 ? sA0 + sb - N : sA0 + sb, s1 = o1 ? sA1 + sb - N : sA1 + sb;
                    const bool w0 = s0 < A.rem, w1 = s1 < A.rem;
                    double c;
                    x0s[i] = dsplit(x0s[i] + carr[(rg - 1) * C + b], w0 ? iv1 : iv0, w0 ? pw1 : pw0, c);
                    x1s[i] = dsplit(x1s[i] + c, w1 ? iv1 : iv0, w1 ? pw1 : pw0, c);
                    carr2[rg * C + b] = c;
                }
            }
            if (ph == 0) {
                // row R-1, column b feeds row 0, column b+1; column C-1 wraps to digit 0
                if (rg == G - 1) {
#pragma unroll
                    for (int i = 0; i < E; ++i) {
                        const int b = tr + TR * i;
                        hin[(b + 1) & (C - 1)] = carr[(G - 1) * C + b];
                        hin2[(b + 1) & (C - 1)] = carr2[(G - 1) * C + b];
                    }
                }
                __syncthreads();  // carry arrays read before phase 1 reloads the buffers
                continue;
            }
            if (rg == G - 1) {
#pragma unroll
                for (int i = 0; i < E; ++i) {
                    const int b = tr + TR * i;
                    A.carry[(size_t)blk * C + b] = carr[(G - 1) * C + b];
                    A.carry2[(size_t)blk * C + b] = (float)carr2[(G - 1) * C + b];
                }
                __threadfence();  // each writer orders its carry-out stores before the flag below
            }
            __syncthreads();
            // ---- hop 3 for rows 2 .. G-1: the small second-digit carry of the row above ----
            if (rg >= 2) {
#pragma unroll
                for (int i = 0; i < E; ++i) x0s[i] += carr2[(rg - 1) * C + tr + TR * i];
            }
            if (t == 0) {
                __threadfence();
                *reinterpret_cast<volatile unsigned*>(&A.flags[blk]) = ep + 1u;
                const unsigned long long eb = s_err;
                atomicMax(&A.ctl->err_max, eb);
                atomicMax(&A.ctl->err_since, eb);
                if (A.errlog) atomicMax(reinterpret_cast<unsigned int*>(A.errlog + (ep % (unsigned)A.errlog_len)),
                                        __float_as_uint((float)__longlong_as_double((long long)eb)));
            }
            // The carry arrays are read: each row may now reuse its exchange buffer, and rows
            // 2 .. G-1 go on to the forward FFT. Row 0 waits for the previous block's carry-outs
            // (hop 2 and 3 from outside the block); row 1 waits for row 0's hop-2 carry-outs,
            // which pass through `late` (outside the exchange buffers).
            __syncthreads();
            if constexpr (TR >= 32) {
                if (rg == 0) {
                    if (t == 0 && blk > 0) wait_flag(&A.flags[blk - 1], ep + 1u, A.ctl, kSpinLimit);
                    NamedSync{1u, (unsigned)TR}();
                }
            } else {
                if (t == 0 && blk > 0) wait_flag(&A.flags[blk - 1], ep + 1u, A.ctl, kSpinLimit);
                __syncthreads();
            }
            // ---- hop 2 and 3 for the block's first row: previous block's last row, or the wrap ----
            if (rg == 0) {
#pragma unroll
                for (int i = 0; i < E; ++i) {
                    const int b = tr + TR * i;
                    double cin = (blk > 0) ? __ldcg(A.carry + (size_t)(blk - 1) * C + b) : hin[b];
                    if (a == 0 && b == 0) cin -= 2.0;  // the "- 2" of s^2 - 2 (digit 0)
                    const int sb = sB_of(b);
                    const bool o0 = sA0 + sb >= N, o1 = sA1 + sb >= N;
                    const int s0 = o0 ? sA0 + sb - N : sA0 + sb, s1 = o1 ? sA1 + sb - N : sA1 + sb;
                    const bool w0 = s0 < A.rem, w1 = s1 < A.rem;
                    double c;
                    x0s[i] = dsplit(x0s[i] + cin, w0 ? iv1 : iv0, w0 ? pw1 : pw0, c);
                    x1s[i] = dsplit(x1s[i] + c, w1 ? iv1 : iv0, w1 ? pw1 : pw0, c);
                    late[b] = c;
                    x0s[i] += (blk > 0) ? (double)__ldcg(A.carry2 + (size_t)(blk - 1) * C + b) : hin2[b];
                }
            }
            if constexpr (TR >= 32) {
                if (rg == 0) {
                    __threadfence_block();
                    NamedSync{(unsigned)G + 1u, 2u * TR}.arrive();
                } else if (rg == 1) {
                    NamedSync{(unsigned)G + 1u, 2u * TR}();
                }
            } else {
                __syncthreads();
            }
            // ---- hop 3 for row 1 ----
            if (rg == 1) {
#pragma unroll
                for (int i = 0; i < E; ++i) x0s[i] += late[tr + TR * i];
            }
            if (MODE == LARGE_FINAL || A.dump) {
#pragma unroll
                for (int i = 0; i < E; ++i) {
                    const int b = tr + TR * i;
                    const size_t m = (size_t)a + (size_t)R * b;
                    *reinterpret_cast<int2*>(A.digits + 2 * m) =
                        make_int2(__double2int_rn(x0s[i]), __double2int_rn(x1s[i]));
                }
            }
        }
        if constexpr (MODE == LARGE_FINAL) return;
    }

    // ---- weight, forward row FFT, store ----
    const int sA0 = __ldg(A.sA + 2 * a), sA1 = __ldg(A.sA + 2 * a + 1);
    const double wa0 = __ldg(A.wA + 2 * a), wa1 = __ldg(A.wA + 2 * a + 1);
#pragma unroll
    for (int i = 0; i < E; ++i) {
        const int b = tr + TR * i;
        const int sb = sB_of(b);
        const double wb = __ldg(A.wB + b);
        const bool o0 = sA0 + sb >= N, o1 = sA1 + sb >= N;
        v[i].x = x0s[i] * (wa0 * wb) * (o0 ? 0.5 : 1.0);
        v[i].y = x1s[i] * (wa1 * wb) * (o1 ? 0.5 : 1.0);
    }
    forward_from<GC, 0>(v, buf, qtw, tr, gsync);
#pragma unroll
    for (int j = 0; j < E; ++j) buf[phys(tr * E + j)] = v[j];
    if (MODE == LARGE_ITER && blk == A.nblocks - 1 && t == 0) {
        // rows R-G .. R-1 are block 0's wrap-around input: wait (bounded) until it has read them
        wait_flag(&A.ctl->halo_read, ep + 1u, A.ctl, kSpinLimit);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < G * C / T; ++r) {
        const int qq = t + T * r, pos = qq / G, ra = qq % G;
        A.V[(size_t)pos * R + a0 + ra] = bufs[ra * RS + phys(pos)];
    }
}

// Column pass: one block owns the column pair (c, C-c), one half of its threads per column; the
// real-FFT split reads the partner column's spectrum from the other half's exchange buffer.
// Block 0 holds column 0 and block C/2 column C/2, each of which pairs with itself.
template <int LOG_R>
__global__ void __launch_bounds__(2 * (1 << LOG_R) / (1 << kLargeLogE), (LOG_R <= 11 ? 2 : 1)) large_col(const LargeArgs A) {
    using GR = SmallG<LOG_R, kLargeLogE>;
    constexpr int R = GR::M, TC = GR::T, E = GR::E;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* bufs = reinterpret_cast<double2*>(smem_raw);  // 2 exchange buffers of PAD slots
    double2* qtw = bufs + 2 * GR::PAD;                       // padded quarter table (R-point)
    constexpr int QL = (int)qpad_len(R / 4);
    const int t = threadIdx.x, half = t / TC, tc = t % TC;
    const int C = A.C;
    const int cb = blockIdx.x;  // 0 .. C/2
    const int c1 = cb, c2 = (C - cb) & (C - 1);
    const bool self = (c1 == c2);
    const bool active = !(self && half == 1);
    const int c = half ? c2 : c1;
    double2* buf = bufs + half * GR::PAD;
    const double2* pbuf = self ? buf : bufs + (1 - half) * GR::PAD;  // partner column
    // each column's FFT exchanges wait only on that column's warps (named barrier 1 + half)
    using ColSync = typename std::conditional<(TC >= 32), NamedSync, CtaSync>::type;
    ColSync gsync;
    if constexpr (TC >= 32) gsync = NamedSync{1u + (unsigned)half, (unsigned)TC};
    for (int k = t; k < QL; k += 2 * TC) qtw[k] = A.qtwR[k];
    double2* col = A.V + (size_t)__ldg(A.pos_of_c + c) * R;
    // four-step twiddle w_M^{a c} for a = tc + TC i, factored as w_M^{c tc} * w_M^{c TC i}: one
    // value per thread and an E-entry table per column (broadcast reads)
    double2* ptab = qtw + QL + half * E;
    for (int i = tc; i < E; i += TC) ptab[i] = twiddle_M(A, (uint32_t)c * (uint32_t)(TC * i), false);
    const double2 q = twiddle_M(A, (uint32_t)c * (uint32_t)tc, false);
    double2 v[E];
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = active ? col[tc + TC * i] : make_double2(0.0, 0.0);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = cmul(v[i], cmul(q, ptab[i]));
    forward_from<GR, 0>(v, buf, qtw, tc, gsync);
#pragma unroll
    for (int j = 0; j < E; ++j) buf[phys(tc * E + j)] = v[j];
    __syncthreads();
    const double2 wc = __ldg(A.tw1 + c);  // w_M^c
#pragma unroll
    for (int j = 0; j < E; ++j) {
        const int d = freq_of_pos<GR>(tc * E + j);
        const int dp = (c == 0) ? ((R - d) & (R - 1)) : (R - 1 - d);
        const int xp = phys(pos_of_freq<GR>(dp));
        const double2 Av = v[j], Bc = conj2(pbuf[xp]);  // conj(U_{M-k})
        const double2 s = cadd(Av, Bc), dd = csub(Av, Bc);
        const double2 a3 = make_double2(3.0 * Av.x - Bc.x, 3.0 * Av.y - Bc.y);
        const double2 d2 = make_double2((dd.x - dd.y) * (dd.x + dd.y), 2.0 * dd.x * dd.y);
        const double2 w = cmul(wc, twiddle<LOG_R>(qtw, (uint32_t)d, false));  // w_M^{c + C d}
        v[j] = csub(cmul(a3, s), cmul(w, d2));
    }
    __syncthreads();  // partner reads done before either column overwrites its buffer
    inverse_from<GR, GR::P - 1, false>(v, buf, qtw, tc, gsync);
    if (active) {
        const double2 q2 = twiddle_M(A, (uint32_t)c * (uint32_t)tc, false);  // recomputed: frees registers
#pragma unroll
        for (int i = 0; i < E; ++i) col[tc + TC * i] = cmulc(v[i], cmul(q2, ptab[i]));
    }
    if (cb == 0 && t == 0) atomicAdd(&A.ctl->epoch, 1u);
}

template <int LOG_C, int G>
static size_t row_smem() {
    using GC = SmallG<LOG_C, large_row_log_e(LOG_C, G), TW_FULL>;
    return sizeof(double2) * (G * (GC::PAD + 1) + twiddle_table_len<GC>()) + sizeof(double) * GC::M;
}

template <int LOG_R>
static size_t col_smem() {
    using GR = SmallGeom<LOG_R, kLargeLogE>;
    return sizeof(double2) * 2 * GR::PAD + sizeof(double2) * qpad_len(GR::M / 4) + sizeof(double2) * 2 * GR::E;
}

template <int LOG_C, int G, int MODE>
static cudaError_t row_attr() {
    return cudaFuncSetAttribute(large_row<LOG_C, G, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)row_smem<LOG_C, G>());
}

template <int LOG_C, int G>
static cudaError_t row_attrs() {
    cudaError_t e = row_attr<LOG_C, G, LARGE_INIT>();
    if (!e) e = row_attr<LOG_C, G, LARGE_ITER>();
    if (!e) e = row_attr<LOG_C, G, LARGE_FINAL>();
    return e;
}

template <int LOG_R>
static cudaError_t col_attr() {
    return cudaFuncSetAttribute(large_col<LOG_R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)col_smem<LOG_R>());
}

template <int LOG_C, int G, int MODE>
static cudaError_t row_t(const LargeArgs& a, cudaStream_t st) {
    large_row<LOG_C, G, MODE><<<a.nblocks, large_row_threads(LOG_C, G), row_smem<LOG_C, G>(), st>>>(a);
    return cudaGetLastError();
}

template <int LOG_R>
static cudaError_t col_t(const LargeArgs& a, cudaStream_t st) {
    large_col<LOG_R><<<a.C / 2 + 1, 2 * (1 << LOG_R) / (1 << kLargeLogE), col_smem<LOG_R>(), st>>>(a);
    return cudaGetLastError();
}

// Opts the kernels of one geometry into their dynamic shared memory (once per device, before
// any launch or graph capture).
cudaError_t configure_large(int log_c, int g, int log_r) {
    cudaError_t e = cudaSuccess;
    if (!large_rows_supported(log_c, g)) return cudaErrorInvalidValue;
    const int key = 16 * log_c + g;
    switch (key) {
        case 16 * 6 + 4: e = row_attrs<6, 4>(); break;
        case 16 * 7 + 4: e = row_attrs<7, 4>(); break;
        case 16 * 8 + 4: e = row_attrs<8, 4>(); break;
        case 16 * 9 + 4: e = row_attrs<9, 4>(); break;
        case 16 * 10 + 4: e = row_attrs<10, 4>(); break;
        case 16 * 11 + 4: e = row_attrs<11, 4>(); break;
        case 16 * 8 + 2: e = row_attrs<8, 2>(); break;
        case 16 * 9 + 2: e = row_attrs<9, 2>(); break;
        case 16 * 10 + 2: e = row_attrs<10, 2>(); break;
        case 16 * 11 + 2: e = row_attrs<11, 2>(); break;
        case 16 * 9 + 8: e = row_attrs<9, 8>(); break;
        case 16 * 10 + 8: e = row_attrs<10, 8>(); break;
        default: return cudaErrorInvalidValue;
    }
    if (e) return e;
    switch (log_r) {
        case 7: return col_attr<7>();
        case 8: return col_attr<8>();
        case 9: return col_attr<9>();
        case 10: return col_attr<10>();
        case 11: return col_attr<11>();
        case 12: return col_attr<12>();
        default: return cudaErrorInvalidValue;
    }
}

template <int MODE>
static cudaError_t row_mode(int log_c, int g, const LargeArgs& a, cudaStream_t st) {
    switch (16 * log_c + g) {
        case 16 * 6 + 4: return row_t<6, 4, MODE>(a, st);
        case 16 * 7 + 4: return row_t<7, 4, MODE>(a, st);
        case 16 * 8 + 4: return row_t<8, 4, MODE>(a, st);
        case 16 * 9 + 4: return row_t<9, 4, MODE>(a, st);
        case 16 * 10 + 4: return row_t<10, 4, MODE>(a, st);
        case 16 * 11 + 4: return row_t<11, 4, MODE>(a, st);
        case 16 * 8 + 2: return row_t<8, 2, MODE>(a, st);
        case 16 * 9 + 2: return row_t<9, 2, MODE>(a, st);
        case 16 * 10 + 2: return row_t<10, 2, MODE>(a, st);
        case 16 * 11 + 2: return row_t<11, 2, MODE>(a, st);
        case 16 * 9 + 8: return row_t<9, 8, MODE>(a, st);
        case 16 * 10 + 8: return row_t<10, 8, MODE>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_large_row(int log_c, int g, int mode, const LargeArgs& a, cudaStream_t st) {
    switch (mode) {
        case LARGE_INIT: return row_mode<LARGE_INIT>(log_c, g, a, st);
        case LARGE_ITER: return row_mode<LARGE_ITER>(log_c, g, a, st);
        case LARGE_FINAL: return row_mode<LARGE_FINAL>(log_c, g, a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_large_col(int log_r, const LargeArgs& a, cudaStream_t st) {
    switch (log_r) {
        case 7: return col_t<7>(a, st);
        case 8: return col_t<8>(a, st);
        case 9: return col_t<9>(a, st);
        case 10: return col_t<10>(a, st);
        case 11: return col_t<11>(a, st);
        case 12: return col_t<12>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace llg
