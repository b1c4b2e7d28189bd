// Two-pass FP64 IBDWT squaring for N = 2^14 .. 2^23 with the residue resident in HBM.
//
// The M = N/2 packed complex values u_m (m = a + R*b: row a < R, column b < C, M = R*C) are
// transformed by the four-step method. One squaring is two kernels, i.e. two read+write sweeps of
// the 16*M-byte state -- the fewest a transform of this size allows when each pass's working set
// must fit on chip (the reference does one monolithic FFTW transform per direction,
// lucaslehmer.cpp:283,288, and an O(N) host loop for each of weight, unweight and carry,
// lucaslehmer.cpp:282,289-310):
//
//   row pass (one block = a tile of G consecutive rows, G = 2, 4 or 8, all C columns):
//       inverse C-point FFT                                   (end of the previous squaring)
//       unweight, round, max round-off, carry, "- 2"
//       weight, forward C-point FFT                           (start of this squaring)
//   column pass (one block = the column pair c, C-c):
//       twiddle w_M^{ac}, forward R-point FFT, real-FFT split + pointwise square over the pair
//       (k, M-k), inverse R-point FFT, twiddle w_M^{-ac}
//
// The state is stored column-slot-major (element (a, pos) at pos*R + a), so a row tile reads and
// writes G contiguous complex values (16 G bytes) per column slot and a column block reads and
// writes its columns contiguously.
//
// Row tiles interleave their rows across the lanes of every warp: thread t works on row t % G of
// the tile at FFT thread index t / G. A tile's loads and stores then go straight between HBM and
// registers in runs of 16 G bytes (no shared-memory transpose), the FFT exchange buffer holds
// slot x of row r at physp(x) * G + r (a quarter warp touches one contiguous 16 G-byte run:
// conflict-free), and the carry between the rows of a tile is a shuffle between neighbouring
// lanes.
//
// Carry. Digits 2m, 2m+1 of row a carry into row a+1 (m -> m+1 is a -> a+1), so the chain runs
// down the rows of each column b. Each row's carry-out is computed from that row's rounded values
// alone (two-digit chain started at zero: hop 1); the incoming carry is folded into the first
// digit and split again (hop 2), and the small remainder of that split goes into the next row's
// first digit (hop 3). That keeps every digit within a few units of balanced and makes carry-outs
// independent of carry-ins. Inside a tile the carries pass between lanes; between tiles, tile k
// publishes its last row's hop-1 and hop-2 carry-outs and a flag, and tile k+1 reads them after a
// bounded wait. Tiles take tickets in launch order, so the tile waited on is always resident or
// finished. The wrap-around carry into row 0 (2^p == 1) comes from row R-1: the first ticket is a
// separate job that runs the last tile's rows through the inverse FFT and hops 1-2 and publishes
// their carry-outs (one column on) in the slot tile 0 reads; the last tile waits (bounded) for
// that job before overwriting those rows.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "llg_device.cuh"
#include "llg_fft.cuh"
#include "llg_host.h"
#include "llg_internal.h"

namespace llg {

namespace {

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
    const int b = (large_row_log_e(log_c, g) >= 4 ? 512 : 1024) / large_row_threads(log_c, g);
    return b > 16 ? 16 : (b < 1 ? 1 : b);
}
// exchange-buffer slots of a tile: G rows of C + C/E padded slots
__host__ __device__ constexpr int large_row_slots(int log_c, int g) {
    return g * ((1 << log_c) + ((1 << log_c) >> large_row_log_e(log_c, g)));
}

template <int LOG_C, int G, int MODE>
__global__ void __launch_bounds__(large_row_threads(LOG_C, G), large_row_min_blocks(LOG_C, G))
    large_row(const LargeArgs A) {
    constexpr int LE = large_row_log_e(LOG_C, G);
    using GC = SmallG<LOG_C, LE, TW_FULL, true>;  // full twiddle table, factored twiddles
    constexpr int C = GC::M, TR = GC::T, E = GC::E, T = G * TR;
    static_assert(T % 32 == 0 && 32 % G == 0, "whole warps of whole row groups");
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int QL = (int)twiddle_table_len<GC>();
    double2* xbuf = reinterpret_cast<double2*>(smem_raw);          // exchange: slot physp(x) * G + row
    double2* qtw = xbuf + large_row_slots(LOG_C, G);               // padded twiddle table (C-point)
    double* swB = reinterpret_cast<double*>(qtw + QL);             // C column weights 2^(sB/N)
    double* siwB = swB + C;                                        // C inverse column weights
    int* ssB = reinterpret_cast<int*>(siwB + C);                   // C column weight exponents sB
    __shared__ unsigned long long s_err;
    __shared__ int s_job;
    __shared__ unsigned s_epoch;

    const int t = threadIdx.x, ra = t % G, tr = t / G;
    double2* buf = xbuf + ra;
    const int N = A.N, R = A.R;
    const CtaSync sync;

    // The next pass may launch once every block of this one has started (its blocks then take
    // the SMs this pass's last wave leaves idle). This pass's own constant tables are requested
    // (asynchronous copies, completed before the barrier that follows the tile loads) before it
    // waits for the previous pass to complete; nothing it reads from the state, the control block
    // or the carry slots is touched before that wait.
    pdl_launch_dependents();
    for (int k = t; k < QL; k += T) cp_async<16>(qtw + k, A.qtwC + k);
    for (int k = t; k < C; k += T) {
        cp_async<8>(swB + k, A.wB + k);
        if (MODE != LARGE_INIT) cp_async<8>(siwB + k, A.iwB + k);
        cp_async<4>(ssB + k, A.sB + k);
    }
    pdl_wait_previous();

    if (t == 0) {
        const unsigned ep = *reinterpret_cast<volatile unsigned*>(&A.ctl->epoch);
        s_epoch = ep;
        if (MODE == LARGE_INIT) {
            s_job = blockIdx.x;
        } else {
            // tickets in launch order: ticket 0 is the wrap-around job, ticket k tile k - 1
            const int tk = (int)atomicAdd(&A.ctl->ticket[ep & 1], 1u);
            if (tk == A.nblocks) {
                // every block of this launch holds its ticket: both counters can be reset
                A.ctl->ticket[(ep + 1) & 1] = 0u;
                A.ctl->ticket[ep & 1] = 0u;
            }
            s_job = tk - 1;
        }
        s_err = 0ull;
    }
    __syncthreads();
    const int job = s_job;  // -1: the wrap-around job (rows R-G .. R-1), else the tile
    const unsigned ep = s_epoch;
    const bool wrap_job = job < 0;
    const int a = (wrap_job ? R - G : job * G) + ra;  // this thread's row
    // weight exponent s = (sA(2a+e) + sB(b)) mod N of digit 2m+e, sB(b) = (-2 R b p) mod N from
    // the shared-memory copy of its table. digit_kind(b) gives bit 0 / 1: digit 0 / 1 of (a, b) has
    // q + 1 bits (s < p mod N); bit 2 / 3: sA + sB wrapped past N, so the weight 2^(s/N) is the
    // table product times 1/2 (and the inverse weight times 2). Recomputed where used: a few
    // integer operations, fewer live registers than keeping them.
    const int sA0 = __ldg(A.sA + 2 * a), sA1 = __ldg(A.sA + 2 * a + 1);
    auto kind_at = [&](int s0a, int s1a, int b) {
        const int sb = ssB[b];
        const bool o0 = s0a + sb >= N, o1 = s1a + sb >= N;
        const int s0 = o0 ? s0a + sb - N : s0a + sb, s1 = o1 ? s1a + sb - N : s1a + sb;
        return (uint32_t)(s0 < A.rem) | ((uint32_t)(s1 < A.rem) << 1) | ((uint32_t)o0 << 2) | ((uint32_t)o1 << 3);
    };
    auto digit_kind = [&](int b) { return kind_at(sA0, sA1, b); };
    // the digit kinds of this thread's E values, 4 bits each, from the carry to the re-weighting
    // (at 16 values a thread; at 8, where registers are scarcer, recomputed)
    constexpr bool KEEP_KINDS = LE >= 4;
    uint32_t kinds[(E + 7) / 8];
#pragma unroll
    for (int w = 0; w < (E + 7) / 8; ++w) kinds[w] = 0u;

    double2 v[E];
    if constexpr (MODE == LARGE_INIT) {
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const size_t m = (size_t)a + (size_t)R * (tr + TR * i);
            const int2 d = *reinterpret_cast<const int2*>(A.digits + 2 * m);
            v[i] = make_double2((double)d.x, (double)d.y);
        }
        cp_async_wait_all();
        __syncthreads();  // the tables are in shared memory
    } else {
        // ---- the tile's rows, straight into registers: thread (row, tr) holds positions
        //      tr E .. tr E + E-1 (the forward FFT's output order), G rows per 16 G-byte run ----
        {
            const double2* lp = A.V + (size_t)(tr * E) * R + a;
#pragma unroll
            for (int j = 0; j < E; ++j) v[j] = __ldcg(lp + (size_t)j * R);
        }
        cp_async_wait_all();
        __syncthreads();  // the tables are in shared memory
        inverse_from<GC, GC::P - 1, false, CtaSync, G, LE>(v, buf, qtw, tr, sync);

        // ---- hop 1: unweight, round, round-off, two-digit chain from zero; hop 2 for rows fed
        //      from inside the tile (the carry-out of the lane above); hop 3 for rows 2 .. G-1 (the
        //      hop-2 carry-out of the row above, also known inside the tile). Row G-1 publishes its
        //      hop-1 and hop-2 carry-outs for the next tile (the wrap job: one column on). ----
        const int slot = job + 1;
        const double ia0 = __ldg(A.iwA + 2 * a), ia1 = __ldg(A.iwA + 2 * a + 1);
        double lerr = 0.0;
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int b = tr + TR * i;
            const double iwb = siwB[b];
            const uint32_t kd = digit_kind(b);
            if (KEEP_KINDS) kinds[i / 8] |= kd << (4 * (i % 8));
            const int w0 = kd & 1u, w1 = (kd >> 1) & 1u;
            const double va = v[i].x * (ia0 * iwb) * ((kd & 4u) ? 2.0 : 1.0);
            const double vb = v[i].y * (ia1 * iwb) * ((kd & 8u) ? 2.0 : 1.0);
            long long ia, ib;
            const double r0 = round_shift(va, ia), r1 = round_shift(vb, ib);
            lerr = fmax(lerr, fmax(fabs(va - r0), fabs(vb - r1)));
            double c, c1, c2 = 0.0;
            double x0 = dsplit_e(r0, A.q + w0, c);
            double x1 = dsplit_e(r1 + c, A.q + w1, c1);
            const double cin = __shfl_up_sync(FULL, c1, 1, G);
            if (ra > 0) {
                x0 = dsplit_e(x0 + cin, A.q + w0, c);
                x1 = dsplit_e(x1 + c, A.q + w1, c2);
            }
            const double cin2 = __shfl_up_sync(FULL, c2, 1, G);
            if (ra > 1) x0 += cin2;
            if (ra == G - 1) {
                const int col = wrap_job ? ((b + 1) & (C - 1)) : b;  // row R-1, column b feeds row 0, column b+1
                A.carry[(size_t)slot * C + col] = c1;
                A.carry2[(size_t)slot * C + col] = c2;
            }
            v[i] = make_double2(x0, x1);
        }
        // the tile's round-off max: one shared atomic per warp
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lerr = fmax(lerr, __shfl_xor_sync(FULL, lerr, o));
        if ((t & 31) == 0) atomicMax(&s_err, (unsigned long long)__double_as_longlong(lerr));
        if (ra == G - 1) __threadfence();  // each publisher orders its carry stores before the flag
        __syncthreads();
        if (t == 0) {
            *reinterpret_cast<volatile unsigned*>(&A.flags[slot]) = ep + 1u;
            if (!wrap_job) {
                const unsigned long long eb = s_err;
                atomicMax(&A.ctl->err_max, eb);
                atomicMax(&A.ctl->err_since, eb);
                if (A.errlog)
                    atomicMax(reinterpret_cast<unsigned int*>(A.errlog + (ep % (unsigned)A.errlog_len)),
                              __float_as_uint((float)__longlong_as_double((long long)eb)));
            }
        }
        if (wrap_job) return;
        // ---- the tile's first row: hops 2 and 3 from the previous tile's last row (or the wrap);
        //      its hop-2 carry-outs are hop 3 of the second row. The row passes through the
        //      exchange buffer (free until the forward FFT's first stores), so that every thread
        //      takes E / G of its columns rather than one lane in G all of them. ----
        double2* row0 = xbuf;                                    // C slots: row 0 of the tile
        double* hop3 = reinterpret_cast<double*>(xbuf + C);      // C doubles: hop 3 into row 1
        if (ra == 0) {
#pragma unroll
            for (int i = 0; i < E; ++i) row0[tr + TR * i] = v[i];
        }
        if (t == 0) wait_flag(&A.flags[job], ep + 1u, A.ctl, A.spin_limit);
        __syncthreads();
        {
            const int a0 = job * G;
            const int s0a = __ldg(A.sA + 2 * a0), s1a = __ldg(A.sA + 2 * a0 + 1);
            const double* cprev = A.carry + (size_t)job * C;
            const double* c2prev = A.carry2 + (size_t)job * C;
            static_assert(C % T == 0, "whole columns per thread");
#pragma unroll
            for (int k = 0; k < C / T; ++k) {
                const int b = t + T * k;
                const uint32_t kd = kind_at(s0a, s1a, b);
                double cin = __ldcg(cprev + b);
                if (job == 0 && b == 0) cin -= 2.0;  // the "- 2" of s^2 - 2 (digit 0)
                const double2 x = row0[b];
                double c, c2;
                const double x0 = dsplit_e(x.x + cin, A.q + (int)(kd & 1u), c);
                const double x1 = dsplit_e(x.y + c, A.q + (int)((kd >> 1) & 1u), c2);
                row0[b] = make_double2(x0 + __ldcg(c2prev + b), x1);
                hop3[b] = c2;
            }
        }
        __syncthreads();
        if (ra == 0) {
#pragma unroll
            for (int i = 0; i < E; ++i) v[i] = row0[tr + TR * i];
        } else if (ra == 1) {
#pragma unroll
            for (int i = 0; i < E; ++i) v[i].x += hop3[tr + TR * i];
        }
        if (MODE == LARGE_FINAL || A.dump) {
#pragma unroll
            for (int i = 0; i < E; ++i) {
                const size_t m = (size_t)a + (size_t)R * (tr + TR * i);
                *reinterpret_cast<int2*>(A.digits + 2 * m) = make_int2(__double2int_rn(v[i].x), __double2int_rn(v[i].y));
            }
        }
        if constexpr (MODE == LARGE_FINAL) return;
    }

    // ---- weight, forward row FFT, store ----
    const double wa0 = __ldg(A.wA + 2 * a), wa1 = __ldg(A.wA + 2 * a + 1);
#pragma unroll
    for (int i = 0; i < E; ++i) {
        const double wb = swB[tr + TR * i];
        const uint32_t kd = (MODE == LARGE_INIT || !KEEP_KINDS) ? digit_kind(tr + TR * i) : (kinds[i / 8] >> (4 * (i % 8)));
        v[i].x *= (wa0 * wb) * ((kd & 4u) ? 0.5 : 1.0);
        v[i].y *= (wa1 * wb) * ((kd & 8u) ? 0.5 : 1.0);
    }
    // the first forward pass stores after a barrier: the first row's carry may still be read from
    // the exchange buffer
    radix_pass<GC, 0, false, true, CtaSync, G, LE>(v, buf, qtw, tr, sync);
    static_assert(GC::P > 1, "at least two row-FFT passes");
    sync();
    forward_from<GC, 1, CtaSync, G, LE>(v, buf, qtw, tr, sync);
    if (MODE == LARGE_ITER && job == A.nblocks - 1) {
        // rows R-G .. R-1 are the wrap job's input: wait (bounded) until it has read them
        if (t == 0) wait_flag(&A.flags[0], ep + 1u, A.ctl, A.spin_limit);
        __syncthreads();
    }
    // the store addresses equal the load addresses; formed again here from an opaque base, so the
    // compiler does not keep sixteen 64-bit addresses live across the whole pass
    double2* vp = A.V + (size_t)(tr * E) * R + a;
    asm volatile("" : "+l"(vp));
#pragma unroll
    for (int j = 0; j < E; ++j) __stcg(vp + (size_t)j * R, v[j]);
}

// Column pass: one block owns the column pair (c, C-c), one half of its threads per column; the
// real-FFT split reads the partner column's spectrum from the other half's exchange buffer.
// Block 0 holds column 0 and block C/2 column C/2, each of which pairs with itself.
template <int LOG_R>
__global__ void __launch_bounds__(2 * (1 << LOG_R) / (1 << kLargeLogE), (LOG_R <= 11 ? 2 : 1)) large_col(const LargeArgs A) {
    // quarter twiddle table in the spread layout (entry r at qpad_s(r)): the strided twiddle reads
    // of the radix passes spread over more bank groups than with qpad
    using GR = SmallG<LOG_R, kLargeLogE, TW_QUARTER_S, true>;
    constexpr int R = GR::M, TC = GR::T, E = GR::E;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* bufs = reinterpret_cast<double2*>(smem_raw);  // 2 exchange buffers of PAD slots
    double2* qtw = bufs + 2 * GR::PAD;                       // padded quarter table (R-point)
    constexpr int QL = (int)qpad_s_len(R / 4);
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
    // as in the row pass: the next pass may launch once every block has started; the constant
    // tables are read before waiting for the previous pass
    pdl_launch_dependents();
    for (int k = t; k < QL; k += 2 * TC) qtw[k] = A.qtwR[k];
    double2* col = A.V + (size_t)__ldg(A.pos_of_c + c) * R;
    // four-step twiddle w_M^{a c} for a = tc + TC i, factored as w_M^{c tc} * w_M^{c TC i}: one
    // value per thread and an E-entry table per column (broadcast reads)
    double2* ptab = qtw + QL + half * E;
    for (int i = tc; i < E; i += TC) ptab[i] = twiddle_M(A, (uint32_t)c * (uint32_t)(TC * i), false);
    const double2 q = twiddle_M(A, (uint32_t)c * (uint32_t)tc, false);
    pdl_wait_previous();
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
    // w_M^{c + C d} for the column frequency d of position tc E + j: w_M^c times one table value
    // w_R^{freq_rev} per j / RLAST, times the exact rotation w_RLAST^(j % RLAST)
    const double2 wc = __ldg(A.tw1 + c);  // w_M^c
    constexpr int RL = GR::RLAST, NB = E / RL;
    double2 wk[NB];
#pragma unroll
    for (int h = 0; h < NB; ++h) wk[h] = cmul(wc, twiddle<LOG_R, true>(qtw, (uint32_t)freq_rev<GR>(tc * NB + h), false));
#pragma unroll
    for (int j = 0; j < E; ++j) {
        const int d = freq_of_pos<GR>(tc * E + j);
        const int dp = (c == 0) ? ((R - d) & (R - 1)) : (R - 1 - d);
        const int xp = phys(pos_of_freq<GR>(dp));
        const double2 Av = v[j], Bc = conj2(pbuf[xp]);  // conj(U_{M-k})
        const double2 s = cadd(Av, Bc), dd = csub(Av, Bc);
        const double2 a3 = make_double2(3.0 * Av.x - Bc.x, 3.0 * Av.y - Bc.y);
        const double2 d2 = make_double2((dd.x - dd.y) * (dd.x + dd.y), 2.0 * dd.x * dd.y);
        v[j] = csub(cmul(a3, s), cmul(wk[j / RL], rot_k<RL, false>(d2, j % RL)));
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

// e^{-2 pi i x / R} (conjugated when inv) for x < R, R a multiple of 4, from the padded quarter
// table of R points (R need not be a power of two).
template <int R>
__device__ __forceinline__ double2 twiddle_r(const double2* __restrict__ q, uint32_t x, bool inv) {
    constexpr uint32_t QR = (uint32_t)R / 4;
    const uint32_t quad = x / QR;
    const double2 w = q[qpad(x - quad * QR)];
    double2 r;
    switch (quad & 3u) {
        case 0: r = w; break;
        case 1: r = make_double2(w.y, -w.x); break;
        case 2: r = make_double2(-w.x, -w.y); break;
        default: r = make_double2(-w.y, w.x); break;
    }
    return inv ? conj2(r) : r;
}

// acc + a w + b conj(w): the radix-R0 terms of r and R0 - r share their factor up to conjugation.
__device__ __forceinline__ double2 pair_term_r(double2 acc, double2 a, double2 b, double2 w) {
    const double sx = a.x + b.x, sy = a.y + b.y, dx = a.x - b.x, dy = a.y - b.y;
    return make_double2(fma(-dy, w.y, fma(sx, w.x, acc.x)), fma(dx, w.y, fma(sy, w.x, acc.y)));
}

// Column pass at the non-power-of-two column lengths R = R0 L (R0 = 3 or 5, L = 2^LOG_L, 16 values
// per thread), for the {3, 5} x 2^k transform lengths of the reference (lucaslehmer.cpp:244-254).
// One block owns the column pair (c, C-c) as in large_col; each column is split as R0 x L by
// decimation in frequency (a = n + L r, d = R0 k' + k0):
//   U[R0 k' + k0] = sum_n w_L^{n k'} w_R^{n k0} sum_r u[n + L r] w_R0^{r k0}
// the radix-R0 step across the column's R0 segments, the twiddle w_R^{n k0}, R0 L-point FFTs
// (one segment of L/16 threads each, a named barrier per segment), the real-FFT split and square
// over the pair, and back. Thread (half, seg, tl) holds u[seg L + tl + TL i] of its column.
template <int R0, int LOG_L>
__global__ void __launch_bounds__(2 * R0 * (1 << LOG_L) / (1 << kLargeLogE), (2 * R0 * (1 << LOG_L) / (1 << kLargeLogE) <= 256 ? 2 : 1))
    large_col_mixed(const LargeArgs A) {
    using GL = SmallG<LOG_L, kLargeLogE, TW_QUARTER, true>;
    constexpr int L = GL::M, TL = GL::T, E = GL::E, R = R0 * L, TC = R0 * TL, PADL = GL::PAD;
    constexpr int QLL = (int)qpad_len(L / 4), QLR = (int)qpad_len(R / 4);
    static_assert(TL % 32 == 0 && 2 * TC <= 1024, "whole warps per segment");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* bufs = reinterpret_cast<double2*>(smem_raw);  // [half][seg] exchange buffers of PADL slots
    double2* qtwL = bufs + 2 * R0 * PADL;                    // L-point quarter table
    double2* qtwR = qtwL + QLL;                              // R-point quarter table
    double2* omf = qtwR + QLR;                               // [k0][r] w_R0^{r k0}
    double2* omi = omf + R0 * R0;                            // [r][k0] w_R0^{-r k0}
    double2* ptabs = omi + R0 * R0;                          // [half][E] w_M^{c TL i}
    const int t = threadIdx.x, half = t / TC, th = t % TC, seg = th / TL, tl = th % TL;
    const int C = A.C;
    const int cb = blockIdx.x;  // 0 .. C/2
    const int c1 = cb, c2 = (C - cb) & (C - 1);
    const bool self = (c1 == c2);
    const bool active = !(self && half == 1);
    const int c = half ? c2 : c1;
    double2* hb = bufs + half * R0 * PADL;                  // this column's R0 segment buffers
    double2* mybuf = hb + seg * PADL;
    const double2* pb = self ? hb : bufs + (1 - half) * R0 * PADL;  // the partner column's buffers
    // barriers: 1 + half for the column's threads, 3 + half R0 + seg for one segment's
    const NamedSync hsync{1u + (unsigned)half, (unsigned)TC};
    const NamedSync ssync{3u + (unsigned)(half * R0 + seg), (unsigned)TL};
    pdl_launch_dependents();  // as in large_col: constant tables before the wait
    for (int k = t; k < QLL; k += 2 * TC) qtwL[k] = A.qtwL[k];
    for (int k = t; k < QLR; k += 2 * TC) qtwR[k] = A.qtwR[k];
    if (t < R0 * R0) {
        // w_R0^{e}, e = (r k0) mod R0, from the R-point table (R / R0 = L)
        const int x = t / R0, y = t % R0;
        const uint32_t e = (uint32_t)((x * y) % R0) * (uint32_t)L;
        omf[t] = twiddle_r<R>(A.qtwR, e, false);  // [k0 = x][r = y]
        omi[t] = twiddle_r<R>(A.qtwR, e, true);   // [r = x][k0 = y]
    }
    double2* col = A.V + (size_t)__ldg(A.pos_of_c + c) * R;
    // four-step twiddle w_M^{a c}, a = seg L + tl + TL i: w_M^{c (seg L + tl)} w_M^{c TL i}
    double2* ptab = ptabs + half * E;
    for (int i = th; i < E; i += TC) ptab[i] = twiddle_M(A, (uint32_t)c * (uint32_t)(TL * i), false);
    const uint32_t a0 = (uint32_t)(seg * L + tl);
    const double2 q = twiddle_M(A, (uint32_t)c * a0, false);
    pdl_wait_previous();
    double2 v[E];
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = active ? col[a0 + TL * i] : make_double2(0.0, 0.0);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = cmul(v[i], cmul(q, ptab[i]));
    // ---- radix-R0 step across the column's segments, then the twiddle w_R^{n k0} (k0 = seg) ----
#pragma unroll
    for (int i = 0; i < E; ++i) mybuf[phys(tl + TL * i)] = v[i];
    hsync();
#pragma unroll
    for (int i = 0; i < E; ++i) {
        const int n = tl + TL * i;
        double2 acc = hb[phys(n)];
#pragma unroll
        for (int r = 1; 2 * r < R0; ++r) acc = pair_term_r(acc, hb[r * PADL + phys(n)], hb[(R0 - r) * PADL + phys(n)], omf[seg * R0 + r]);
        v[i] = cmul(acc, twiddle_r<R>(qtwR, (uint32_t)(n * seg), false));
    }
    hsync();  // every segment read before the L-point FFTs overwrite the buffers
    forward_from<GL, 0>(v, mybuf, qtwL, tl, ssync);
#pragma unroll
    for (int j = 0; j < E; ++j) mybuf[phys(tl * E + j)] = v[j];
    __syncthreads();
    // ---- real-FFT split + square over the pair: frequency d = R0 kk + k0 of this column pairs with
    //      R - 1 - d of column C - c (c == 0: (R - d) mod R of itself) ----
    {
        const double2 wc = __ldg(A.tw1 + c);  // w_M^c
        constexpr int RL = GL::RLAST, NB = E / RL;
        // w_M^{c + C d} = w_M^c w_R^{k0} w_L^{kk}: one table value per j / RL, times w_RL^(j % RL)
        const double2 wck = cmul(wc, twiddle_r<R>(qtwR, (uint32_t)seg, false));
        double2 wk[NB];
#pragma unroll
        for (int h = 0; h < NB; ++h) wk[h] = cmul(wck, twiddle<LOG_L>(qtwL, (uint32_t)freq_rev<GL>(tl * NB + h), false));
#pragma unroll
        for (int j = 0; j < E; ++j) {
            const int kk = freq_of_pos<GL>(tl * E + j);
            int kp, sp;
            if (c == 0) {
                const int d = R0 * kk + seg;
                const int dp = d == 0 ? 0 : R - d;
                kp = dp / R0;
                sp = dp - R0 * kp;
            } else {
                kp = L - 1 - kk;
                sp = R0 - 1 - seg;
            }
            const int x = sp * PADL + phys(pos_of_freq<GL>(kp));
            const double2 Av = v[j], Bc = conj2(pb[x]);  // conj(U_{M-k})
            const double2 sm = cadd(Av, Bc), dd = csub(Av, Bc);
            const double2 a3 = make_double2(3.0 * Av.x - Bc.x, 3.0 * Av.y - Bc.y);
            const double2 d2 = make_double2((dd.x - dd.y) * (dd.x + dd.y), 2.0 * dd.x * dd.y);
            v[j] = csub(cmul(a3, sm), cmul(wk[j / RL], rot_k<RL, false>(d2, j % RL)));
        }
    }
    __syncthreads();  // partner reads done before either column overwrites its buffers
    inverse_from<GL, GL::P - 1, false>(v, mybuf, qtwL, tl, ssync);
    // ---- conjugate twiddle and the inverse radix-R0 step: thread (r = seg, tl) gets
    //      u[n + L r] = sum_k0 w_R0^{-r k0} w_R^{-n k0} z[k0][n] ----
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = cmul(v[i], twiddle_r<R>(qtwR, (uint32_t)((tl + TL * i) * seg), true));
    ssync();  // this segment's last inverse pass read its buffer
#pragma unroll
    for (int i = 0; i < E; ++i) mybuf[phys(tl + TL * i)] = v[i];
    hsync();
#pragma unroll
    for (int i = 0; i < E; ++i) {
        const int n = tl + TL * i;
        double2 acc = hb[phys(n)];
#pragma unroll
        for (int k0 = 1; 2 * k0 < R0; ++k0)
            acc = pair_term_r(acc, hb[k0 * PADL + phys(n)], hb[(R0 - k0) * PADL + phys(n)], omi[seg * R0 + k0]);
        v[i] = acc;
    }
    if (active) {
        const double2 q2 = twiddle_M(A, (uint32_t)c * a0, false);  // recomputed: frees registers
#pragma unroll
        for (int i = 0; i < E; ++i) col[a0 + TL * i] = cmulc(v[i], cmul(q2, ptab[i]));
    }
    if (cb == 0 && t == 0) atomicAdd(&A.ctl->epoch, 1u);
}

template <int LOG_C, int G>
static size_t row_smem() {
    using GC = SmallG<LOG_C, large_row_log_e(LOG_C, G), TW_FULL, true>;
    return sizeof(double2) * (large_row_slots(LOG_C, G) + twiddle_table_len<GC>()) + (2 * sizeof(double) + sizeof(int)) * GC::M;
}

template <int LOG_R>
static size_t col_smem() {
    using GR = SmallGeom<LOG_R, kLargeLogE>;
    return sizeof(double2) * 2 * GR::PAD + sizeof(double2) * qpad_s_len(GR::M / 4) + sizeof(double2) * 2 * GR::E;
}

// Shared-memory carve-out (percent of the SM's 228 KB) for `blocks` resident blocks of `bytes`
// dynamic shared memory each: no more than they need, so the rest of the on-chip memory stays L1
// (register spills and the weight-table reads hit there).
static int carveout_pct(size_t bytes, int blocks) {
    const size_t need = (size_t)blocks * (bytes + 1024 + 64);  // + the per-block reservation and statics
    const int pct = (int)((100 * need + 228 * 1024 - 1) / (228 * 1024));
    return pct > 100 ? 100 : pct;
}

template <int R0, int LOG_L>
static size_t col_mixed_smem() {
    using GL = SmallGeom<LOG_L, kLargeLogE>;
    constexpr int L = GL::M, R = R0 * L;
    return sizeof(double2) * (2 * R0 * GL::PAD + qpad_len(L / 4) + qpad_len(R / 4) + 2 * R0 * R0 + 2 * GL::E);
}

template <int R0, int LOG_L>
constexpr int col_mixed_threads() { return 2 * R0 * (1 << LOG_L) / (1 << kLargeLogE); }

template <int LOG_C, int G, int MODE>
static cudaError_t row_attr() {
    cudaError_t e = cudaFuncSetAttribute(large_row<LOG_C, G, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)row_smem<LOG_C, G>());
    if (!e)
        e = cudaFuncSetAttribute(large_row<LOG_C, G, MODE>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 carveout_pct(row_smem<LOG_C, G>(), large_row_min_blocks(LOG_C, G)));
    return e;
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
    cudaError_t e = cudaFuncSetAttribute(large_col<LOG_R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)col_smem<LOG_R>());
    if (!e)
        e = cudaFuncSetAttribute(large_col<LOG_R>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 carveout_pct(col_smem<LOG_R>(), LOG_R <= 11 ? 2 : 1));
    return e;
}

template <int R0, int LOG_L>
static cudaError_t col_mixed_attr() {
    cudaError_t e = cudaFuncSetAttribute(large_col_mixed<R0, LOG_L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)col_mixed_smem<R0, LOG_L>());
    if (!e)
        e = cudaFuncSetAttribute(large_col_mixed<R0, LOG_L>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 carveout_pct(col_mixed_smem<R0, LOG_L>(), col_mixed_threads<R0, LOG_L>() <= 256 ? 2 : 1));
    return e;
}

// Launch with programmatic stream serialisation at the power-of-two lengths: the kernel may start
// while the previous kernel of the stream finishes (griddepcontrol in the kernels orders their
// state accesses after it). At the R0 2^k lengths (logN < 0) it measured slower (5 x 2^18: 37.2 ->
// 40.7 us per squaring, against 154.1 -> 148.9 at 2^23), so those launch plainly and the
// griddepcontrol instructions are no-ops.
template <class... KArgs>
static cudaError_t launch_pdl(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t st,
                              const LargeArgs& a) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = a.logN > 0 ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, a);
}

template <int R0, int LOG_L>
static cudaError_t col_mixed_t(const LargeArgs& a, cudaStream_t st) {
    return launch_pdl(large_col_mixed<R0, LOG_L>, a.C / 2 + 1, col_mixed_threads<R0, LOG_L>(),
                      col_mixed_smem<R0, LOG_L>(), st, a);
}

// INIT: one block per tile. ITER / FINAL: one block more, for the wrap-around job (grid == 0), or
// `grid` blocks.
template <int LOG_C, int G, int MODE>
static cudaError_t row_t(const LargeArgs& a, cudaStream_t st, int grid) {
    if (grid <= 0) grid = a.nblocks + (MODE == LARGE_INIT ? 0 : 1);
    return launch_pdl(large_row<LOG_C, G, MODE>, grid, large_row_threads(LOG_C, G), row_smem<LOG_C, G>(), st, a);
}

template <int LOG_R>
static cudaError_t col_t(const LargeArgs& a, cudaStream_t st) {
    return launch_pdl(large_col<LOG_R>, a.C / 2 + 1, 2 * (1 << LOG_R) / (1 << kLargeLogE), col_smem<LOG_R>(), st, a);
}

// Opts the kernels of one geometry into their dynamic shared memory (once per device, before
// any launch or graph capture).
cudaError_t configure_large(int log_c, int g, int log_r) {
    cudaError_t e = cudaErrorInvalidValue;
    switch (16 * log_c + g) {
#define LLG_ROW_ATTRS(LC, GG) \
    case 16 * LC + GG: e = row_attrs<LC, GG>(); break;
        LLG_ROW_SHAPES(LLG_ROW_ATTRS)
#undef LLG_ROW_ATTRS
        default: return cudaErrorInvalidValue;
    }
    if (e) return e;
    switch (log_r) {
        case large_col_code(3, 9): return col_mixed_attr<3, 9>();
        case large_col_code(5, 9): return col_mixed_attr<5, 9>();
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
static cudaError_t row_mode(int log_c, int g, const LargeArgs& a, cudaStream_t st, int grid) {
    switch (16 * log_c + g) {
#define LLG_ROW_LAUNCH(LC, GG) \
    case 16 * LC + GG: return row_t<LC, GG, MODE>(a, st, grid);
        LLG_ROW_SHAPES(LLG_ROW_LAUNCH)
#undef LLG_ROW_LAUNCH
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_large_row(int log_c, int g, int mode, const LargeArgs& a, cudaStream_t st, int grid) {
    switch (mode) {
        case LARGE_INIT: return row_mode<LARGE_INIT>(log_c, g, a, st, grid);
        case LARGE_ITER: return row_mode<LARGE_ITER>(log_c, g, a, st, grid);
        case LARGE_FINAL: return row_mode<LARGE_FINAL>(log_c, g, a, st, grid);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_large_col(int log_r, const LargeArgs& a, cudaStream_t st) {
    switch (log_r) {
        case large_col_code(3, 9): return col_mixed_t<3, 9>(a, st);
        case large_col_code(5, 9): return col_mixed_t<5, 9>(a, st);
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
