// Whole-test-on-chip FP64 IBDWT Lucas-Lehmer kernel for the non-power-of-two lengths
// N = 2 R0 L, R0 in {3, 5}, L = 2^LOG_L (N = 3072, 5120, 6144, 10240, 12288): the reference's
// {3, 5} x 2^k transform lengths (lucaslehmer.cpp:244-254), which hold the same exponent with up to
// 37.5% fewer points than the next power of two.
//
// Same structure as the power-of-two kernel (llg_small.cu): one block per exponent, the M = R0 L
// packed complex values u_m = y_2m + i y_2m+1 stay on chip for all p - 2 squarings. The M-point
// transform is split as R0 x L (decimation in frequency, m = n + L r, k = R0 k' + k0):
//   X[R0 k' + k0] = sum_n w_L^{n k'} w_M^{n k0} sum_r u[n + L r] w_R0^{r k0}
// so a squaring is: the radix-R0 step across the R0 segments (one shared-memory exchange) with the
// twiddle w_M^{n k0}; R0 independent L-point FFTs (the power-of-two radix passes, one segment of
// L/E threads each, named barriers per segment); the real-FFT split and square on the pair
// (k, M - k), which pairs segment k0 with segment R0 - k0; the inverse L-point FFTs; the conjugate
// twiddle and the inverse radix-R0 step; then unweight, round, carry and weight in registers.
//
// Thread t = seg * TL + tl holds u[seg L + tl + TL i], i < E (8 or 16), between squarings: digit
// order runs across the lanes of a segment, then to the next column i, then to the next segment,
// and wraps from the last digit to digit 0 (2^p == 1). The carry-out of a thread does not depend on its
// carry-in (as in the power-of-two kernel), so one exchange per squaring suffices.
#include <cuda_runtime.h>

#include <cstdint>

#include "llg_device.cuh"
#include "llg_fft.cuh"
#include "llg_internal.h"

namespace llg {

namespace {

// values per thread: 8 (radix-8 passes, twice the warps) where the L-point FFT needs no more
// passes than with 16 (L = 2^9: 8 x 8 x 8 against 16 x 16 x 2), else 16
template <int R0_, int LOG_L, int LE_ = (LOG_L == 9 ? 3 : 4)>
struct MixedGeom {
    using GL = SmallG<LOG_L, LE_, TW_QUARTER, true>;
    static constexpr int R0 = R0_;
    static constexpr int L = GL::M, TL = GL::T, E = GL::E;
    static constexpr int M = R0 * L, N = 2 * M, T = R0 * TL;
    static constexpr int W = T / 32, WL = TL / 32;  // warps, warps per segment
    static constexpr int PADL = GL::PAD;            // exchange slots of one segment
    static constexpr int QLL = (int)qpad_len((uint32_t)L / 4);
    static constexpr int QLM = (int)qpad_len((uint32_t)M / 4);
    static_assert(TL % 32 == 0, "a segment is whole warps");
};

// e^{-2 pi i x / M} (conjugated when inv) for x < M, M a multiple of 4, from the padded quarter
// table of M points.
template <int M>
__device__ __forceinline__ double2 twiddle_m(const double2* __restrict__ q, uint32_t x, bool inv) {
    constexpr uint32_t QM = (uint32_t)M / 4;
    const uint32_t quad = x / QM;
    const double2 w = q[qpad(x - quad * QM)];
    double2 r;
    switch (quad & 3u) {
        case 0: r = w; break;
        case 1: r = make_double2(w.y, -w.x); break;
        case 2: r = make_double2(-w.x, -w.y); break;
        default: r = make_double2(-w.y, w.x); break;
    }
    return inv ? conj2(r) : r;
}

// acc + a w + b conj(w): the radix-R0 terms of r and R0 - r share their factor up to conjugation
// (w_R0^{(R0 - r) k} = conj(w_R0^{r k})), so the pair costs two sums and four multiply-adds.
__device__ __forceinline__ double2 pair_term(double2 acc, double2 a, double2 b, double2 w) {
    const double sx = a.x + b.x, sy = a.y + b.y, dx = a.x - b.x, dy = a.y - b.y;
    return make_double2(fma(-dy, w.y, fma(sx, w.x, acc.x)), fma(dx, w.y, fma(sy, w.x, acc.y)));
}

// blocks per SM the kernel is built for (registers: 65536 / (blocks x threads) a thread)
__host__ __device__ constexpr int mixed_min_blocks(int t, int e) {
    return e == 16 ? (t <= 96 ? 4 : t == 160 ? 3 : t <= 192 ? 2 : 1) : (t <= 192 ? 4 : t <= 320 ? 2 : 1);
}

}  // namespace

template <int R0, int LOG_L>
__global__ void __launch_bounds__(MixedGeom<R0, LOG_L>::T, mixed_min_blocks(MixedGeom<R0, LOG_L>::T, MixedGeom<R0, LOG_L>::E))
    ll_small_fp64_mixed(const SmallJob* __restrict__ jobs, const double2* __restrict__ qtwL_g,
                        const double2* __restrict__ qtwM_g, int64_t* __restrict__ digits_out,
                        SmallResult* __restrict__ results, float* __restrict__ errlog, double abort_err) {
    using MG = MixedGeom<R0, LOG_L>;
    using GL = typename MG::GL;
    constexpr int L = MG::L, TL = MG::TL, E = MG::E, M = MG::M, N = MG::N, T = MG::T, W = MG::W,
                  WL = MG::WL, PADL = MG::PADL, QLL = MG::QLL, QLM = MG::QLM;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* bufs = reinterpret_cast<double2*>(smem_raw);  // R0 segment buffers of PADL slots
    double2* qtwL = bufs + R0 * PADL;                        // L-point quarter table
    double2* qtwM = qtwL + QLL;                              // M-point quarter table
    double2* omf = qtwM + QLM;                               // [k0][r] w_R0^{r k0}
    double2* omi = omf + R0 * R0;                            // [r][k0] w_R0^{-r k0}
    double* wB = reinterpret_cast<double*>(omi + R0 * R0);
    double* iwB = wB + E;
    double* cbuf = iwB + E;                                  // W * E carry-outs of last lanes
    int* sB = reinterpret_cast<int*>(cbuf + W * E);
    unsigned long long* serr = reinterpret_cast<unsigned long long*>(sB + E);  // 2 (8-aligned: E even)

    const int t = threadIdx.x;
    const int seg = t / TL, tl = t % TL;
    const int lane = t & 31, warp = t >> 5, wl = warp % WL;
    unsigned long long t_start = 0;
    if (t == 0) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_start));
    const SmallJob job = jobs[blockIdx.x];
    const uint64_t p = job.p;
    const uint64_t iters = job.iters;
    const int q = (int)(p / (uint64_t)N);
    const int rem = (int)(p % (uint64_t)N);

    for (int k = t; k < QLL; k += T) qtwL[k] = qtwL_g[k];
    for (int k = t; k < QLM; k += T) qtwM[k] = qtwM_g[k];
    if (t < R0 * R0) {
        // w_R0^{e}, e = (r k0) mod R0, exact to the last bit from the M-point table (M/R0 = L)
        const int a = t / R0, b = t % R0;
        const uint32_t e = (uint32_t)((a * b) % R0) * (uint32_t)L;
        omf[t] = twiddle_m<M>(qtwM_g, e, false);  // [k0 = a][r = b]
        omi[t] = twiddle_m<M>(qtwM_g, e, true);   // [r = a][k0 = b]
    }
    for (int i = t; i < E; i += T) {
        // digit j = 2m + e with m = seg L + tl + TL i: s_j = (sA(t, e) + sB(i)) mod N
        const uint64_t s = ((uint64_t)N - ((uint64_t)2 * TL * i * p) % (uint64_t)N) % (uint64_t)N;
        sB[i] = (int)s;
        wB[i] = exp2((double)s / (double)N);
        iwB[i] = exp2(-(double)s / (double)N) / (4.0 * (double)M);
    }
    if (t < 2) serr[t] = 0ull;
    __syncthreads();

    const uint64_t m0 = (uint64_t)seg * L + (uint64_t)tl;
    const int sA0 = (int)(((uint64_t)N - ((2 * m0) * p) % (uint64_t)N) % (uint64_t)N);
    const int sA1 = (int)(((uint64_t)N - ((2 * m0 + 1) * p) % (uint64_t)N) % (uint64_t)N);
    const double wA0 = exp2((double)sA0 / (double)N), wA1 = exp2((double)sA1 / (double)N);
    const double iwA0 = exp2(-(double)sA0 / (double)N), iwA1 = exp2(-(double)sA1 / (double)N);

    // kind of the two digits of column i, fixed for the whole test, 4 bits per column: bit 0 / 1:
    // digit 2m / 2m+1 has q + 1 bits; bit 2 / 3: its weight wrapped past N
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

    // the carry into lane 0 of this warp comes from the last lane of warp `src`, column i - shift
    int src, wrapcol;
    if (wl > 0) {
        src = warp - 1;
        wrapcol = 0;
    } else {
        src = seg * WL + WL - 1;  // same segment, previous column (i > 0)
        wrapcol = 1;
    }
    const int src0 = ((seg + R0 - 1) % R0) * WL + WL - 1;  // i == 0 on a segment's first warp

    double2 v[E];
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = make_double2(0.0, 0.0);
    if (t == 0) v[0].x = 4.0;  // s_0 = 4: digit 0 has weight 1

    const NamedSync gsync{1u + (unsigned)seg, (unsigned)TL};
    double2* mybuf = bufs + seg * PADL;
    double maxerr = 0.0;
    uint64_t it = 0;
    uint32_t status = LLG_ST_OK;
    int x0s[E], x1s[E];

    for (;;) {
        // ---- radix-R0 step across the segments, then twiddle w_M^{n k0} (k0 = seg) ----
#pragma unroll
        for (int i = 0; i < E; ++i) mybuf[phys(tl + TL * i)] = v[i];
        __syncthreads();
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int n = tl + TL * i;
            double2 acc = bufs[phys(n)];
#pragma unroll
            for (int r = 1; 2 * r < R0; ++r)
                acc = pair_term(acc, bufs[r * PADL + phys(n)], bufs[(R0 - r) * PADL + phys(n)], omf[seg * R0 + r]);
            v[i] = cmul(acc, twiddle_m<M>(qtwM, (uint32_t)(n * seg), false));
        }
        __syncthreads();  // every segment read before the L-point FFTs overwrite the buffers
        forward_from<GL, 0>(v, mybuf, qtwL, tl, gsync);

        // ---- pair (k, M - k): real-FFT split + square (result scaled by 4, folded into iwB) ----
#pragma unroll
        for (int j = 0; j < E; ++j) mybuf[phys(tl * E + j)] = v[j];
        __syncthreads();
        {
            const int segp = (seg == 0) ? 0 : R0 - seg;
            // w_M^{R0 kk + seg} with kk = freq_rev(tl NB + j / RL) + (j % RL) L / RL: one table
            // value per j / RL, times the exact rotation w_RL^(j % RL)
            constexpr int RL = GL::RLAST, NB = E / RL;
            double2 wk[NB];
#pragma unroll
            for (int h = 0; h < NB; ++h)
                wk[h] = twiddle_m<M>(qtwM, (uint32_t)(R0 * freq_rev<GL>(tl * NB + h) + seg), false);
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const int kk = freq_of_pos<GL>(tl * E + j);
                const int kp = (seg == 0) ? ((L - kk) & (L - 1)) : (L - 1 - kk);
                const int x = segp * PADL + phys(pos_of_freq<GL>(kp));
                const double2 A = v[j], Bc = conj2(bufs[x]);  // conj(U_{M-k})
                const double2 s = cadd(A, Bc), d = csub(A, Bc);
                const double2 a3 = make_double2(3.0 * A.x - Bc.x, 3.0 * A.y - Bc.y);
                const double2 d2 = make_double2((d.x - d.y) * (d.x + d.y), 2.0 * d.x * d.y);
                v[j] = csub(cmul(a3, s), cmul(wk[j / RL], rot_k<RL, false>(d2, j % RL)));
            }
        }
        __syncthreads();  // partner reads (other segments) done before any segment stores
        inverse_from<GL, GL::P - 1, false>(v, mybuf, qtwL, tl, gsync);

        // ---- conjugate twiddle and the inverse radix-R0 step: thread (r = seg, tl) gets
        //      u[n + L r] = sum_k0 w_R0^{-r k0} w_M^{-n k0} z[k0][n] ----
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = cmul(v[i], twiddle_m<M>(qtwM, (uint32_t)((tl + TL * i) * seg), true));
        gsync();  // this segment's last inverse pass read its buffer (no other segment reads it)
#pragma unroll
        for (int i = 0; i < E; ++i) mybuf[phys(tl + TL * i)] = v[i];
        __syncthreads();
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int n = tl + TL * i;
            double2 acc = bufs[phys(n)];
#pragma unroll
            for (int k0 = 1; 2 * k0 < R0; ++k0)
                acc = pair_term(acc, bufs[k0 * PADL + phys(n)], bufs[(R0 - k0) * PADL + phys(n)], omi[seg * R0 + k0]);
            v[i] = acc;
        }

        // ---- unweight, round, error, carry (as in the power-of-two kernel) ----
        double lerr = 0.0;
        refresh_kinds();
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
            if (lane == 31) cbuf[warp * E + i] = cout;
            const double cin = __shfl_up_sync(0xffffffffu, cout, 1);
            if (lane != 0) {
                x0 = dsplit_e(x0 + cin, b0, c);
                x1s[i] = d2i_exact(x1 + c);
            } else {
                x1s[i] = d2i_exact(x1);
            }
            x0s[i] = d2i_exact(x0);
        }
        maxerr = fmax(maxerr, lerr);
        if (errlog) atomicMax(&serr[it & 1], (unsigned long long)__double_as_longlong(lerr));
        const int bad = __syncthreads_or(lerr > abort_err);
        if (errlog && t == 0) {
            errlog[it] = (float)__longlong_as_double((long long)serr[it & 1]);
            serr[(it + 1) & 1] = 0ull;
        }
        refresh_kinds();
        if (lane == 0) {
#pragma unroll
            for (int i = 0; i < E; ++i) {
                double cin;
                if (!wrapcol) cin = cbuf[src * E + i];
                else cin = (i > 0) ? cbuf[src * E + i - 1] : cbuf[src0 * E + E - 1];
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
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const uint32_t kd = kind(i);
            const double w = wB[i];
            v[i].x = i2d_shift(x0s[i]) * (wA0 * w) * ((kd & 4u) ? 0.5 : 1.0);
            v[i].y = i2d_shift(x1s[i]) * (wA1 * w) * ((kd & 8u) ? 0.5 : 1.0);
        }
    }

    if (digits_out) {
        int64_t* out = digits_out + (size_t)blockIdx.x * N;
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const uint64_t m = m0 + (uint64_t)TL * i;
            out[2 * m] = x0s[i];
            out[2 * m + 1] = x1s[i];
        }
    }
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

// ---- the same transform with the radix-R0 steps in registers ----
//
// Between squarings, and for the radix-R0 steps and the carry, thread t < TA = L / NPT holds
// x[c] = u[t + TA c], c < CA = NPT R0: the NPT columns n = t + TA i of every segment r
// (c = i + NPT r). The radix-R0 DFT of column n is then in one thread's registers;
// one store and one load per value move it to and from the segment-major order of the L-point
// FFTs (thread (seg, tl) holds z[seg][tl + TL i]). The layout above reads R0 values from shared
// memory for every output of each radix-R0 step instead. The digit order m = t + TA c runs
// across the lanes, then to the next column, as in the power-of-two kernel, so the carry is that
// kernel's with TA threads and CA columns. The FFTs' R0 segments take at least TA threads:
// R0 = 5, L = 2^9: 320 threads, 256 of them hold 2 columns; R0 = 3, L = 2^9: 192 threads, 128
// of them hold 4 columns; R0 = 3, L = 2^10 (16 values per FFT thread): 192 threads, 128 of them
// hold 8 columns.
template <int R0_, int LOG_L>
struct MixedRGeom {
    using GL = SmallG<LOG_L, LOG_L == 9 ? 3 : 4, TW_QUARTER, true>;
    static constexpr int R0 = R0_;
    static constexpr int L = GL::M, TL = GL::T, E = GL::E;
    static constexpr int M = R0 * L, N = 2 * M;
    static constexpr int NPT = R0 == 5 ? 2 : (LOG_L == 9 ? 4 : 8);  // columns n per digit thread
    static constexpr int MINB = (R0 == 5 || LOG_L > 9) ? 2 : 4;      // blocks per SM the kernel is built for
    static constexpr int TA = L / NPT, CA = NPT * R0, WA = TA / 32;
    static constexpr int T = R0 * TL, W = T / 32;
    static constexpr int PADL = GL::PAD;
    static constexpr int QLL = (int)qpad_len((uint32_t)L / 4);
    static constexpr int QLM = (int)qpad_len((uint32_t)M / 4);
    static_assert(TA <= T && TA % 32 == 0 && TL % 32 == 0, "digit threads are whole warps of the FFT threads");
};

// R0-point DFT in registers: X[k] = sum_r x[r] om[k R0 + r] (om symmetric, om[k][R0 - r] =
// conj(om[k][r])). The terms of r and R0 - r pair up as (x_r + x_{R0-r}) Re w + i (x_r - x_{R0-r}) Im w,
// and X[R0 - k] differs from X[k] only in the sign of the imaginary-weight half.
template <int R0>
__device__ __forceinline__ void dft_r0(double2 (&x)[R0], const double2* __restrict__ om) {
    constexpr int H = (R0 - 1) / 2;
    double2 sm[H], df[H];
#pragma unroll
    for (int r = 1; r <= H; ++r) {
        sm[r - 1] = cadd(x[r], x[R0 - r]);
        df[r - 1] = csub(x[r], x[R0 - r]);
    }
    double2 x0 = x[0];
#pragma unroll
    for (int r = 0; r < H; ++r) x0 = cadd(x0, sm[r]);
#pragma unroll
    for (int k = 1; k <= H; ++k) {
        double2 a = x[0], b = make_double2(0.0, 0.0);
#pragma unroll
        for (int r = 1; r <= H; ++r) {
            const double2 w = om[k * R0 + r];
            a = make_double2(fma(sm[r - 1].x, w.x, a.x), fma(sm[r - 1].y, w.x, a.y));
            b = make_double2(fma(-df[r - 1].y, w.y, b.x), fma(df[r - 1].x, w.y, b.y));
        }
        x[k] = cadd(a, b);
        x[R0 - k] = csub(a, b);
    }
    x[0] = x0;
}

template <int R0, int LOG_L>
__global__ void __launch_bounds__(MixedRGeom<R0, LOG_L>::T, MixedRGeom<R0, LOG_L>::MINB)
    ll_small_fp64_mixed_r(const SmallJob* __restrict__ jobs, const double2* __restrict__ qtwL_g,
                          const double2* __restrict__ qtwM_g, int64_t* __restrict__ digits_out,
                          SmallResult* __restrict__ results, float* __restrict__ errlog, double abort_err) {
    using MG = MixedRGeom<R0, LOG_L>;
    using GL = typename MG::GL;
    constexpr int L = MG::L, TL = MG::TL, E = MG::E, M = MG::M, N = MG::N, T = MG::T, TA = MG::TA,
                  CA = MG::CA, WA = MG::WA, NPT = MG::NPT, PADL = MG::PADL, QLL = MG::QLL, QLM = MG::QLM;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* bufs = reinterpret_cast<double2*>(smem_raw);  // R0 segment buffers of PADL slots
    double2* qtwL = bufs + R0 * PADL;                        // L-point quarter table
    double2* qtwM = qtwL + QLL;                              // M-point quarter table
    double2* omf = qtwM + QLM;                               // [k0][r] w_R0^{r k0}
    double2* omi = omf + R0 * R0;                            // [r][k0] w_R0^{-r k0}
    double* wB = reinterpret_cast<double*>(omi + R0 * R0);   // CA column weights
    double* iwB = wB + CA;
    double* cbuf = iwB + CA;                                 // WA * CA carry-outs of last lanes
    int* sB = reinterpret_cast<int*>(cbuf + WA * CA);
    unsigned long long* serr = reinterpret_cast<unsigned long long*>(sB + CA);  // 2 (8-aligned: CA even)
    static_assert(CA % 2 == 0, "8-byte alignment of serr");
    // slot of the partner U_{M-k} of position tl E + j of this thread's segment, [j][t]: fixed for
    // the whole test, read in the real-FFT split instead of two digit reversals a value
    unsigned short* pslot = reinterpret_cast<unsigned short*>(serr + 2);  // E * T

    const int t = threadIdx.x;
    const bool holds = t < TA;  // a digit thread (whole warps)
    const int seg = t / TL, tl = t % TL;
    const int lane = t & 31, warp = t >> 5;
    unsigned long long t_start = 0;
    if (t == 0) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_start));
    const SmallJob job = jobs[blockIdx.x];
    const uint64_t p = job.p;
    const uint64_t iters = job.iters;
    const int q = (int)(p / (uint64_t)N);
    const int rem = (int)(p % (uint64_t)N);

    for (int k = t; k < QLL; k += T) qtwL[k] = qtwL_g[k];
    for (int k = t; k < QLM; k += T) qtwM[k] = qtwM_g[k];
    if (t < R0 * R0) {
        const int a = t / R0, b = t % R0;
        const uint32_t e = (uint32_t)((a * b) % R0) * (uint32_t)L;
        omf[t] = twiddle_m<M>(qtwM_g, e, false);
        omi[t] = twiddle_m<M>(qtwM_g, e, true);
    }
    for (int c = t; c < CA; c += T) {
        // digit j = 2m + e with m = t + TA c: s_j = (sA(t, e) + sB(c)) mod N
        const uint64_t s = ((uint64_t)N - ((uint64_t)2 * TA * c * p) % (uint64_t)N) % (uint64_t)N;
        sB[c] = (int)s;
        wB[c] = exp2((double)s / (double)N);
        iwB[c] = exp2(-(double)s / (double)N) / (4.0 * (double)M);
    }
    if (t < 2) serr[t] = 0ull;
    {
        const int sg = t / TL, tq = t % TL, sgp = (sg == 0) ? 0 : R0 - sg;
#pragma unroll
        for (int j = 0; j < E; ++j) {
            const int kk = freq_of_pos<GL>(tq * E + j);
            const int kp = (sg == 0) ? ((L - kk) & (L - 1)) : (L - 1 - kk);
            pslot[j * T + t] = (unsigned short)(sgp * PADL + phys(pos_of_freq<GL>(kp)));
        }
    }
    __syncthreads();

    const int sA0 = (int)(((uint64_t)N - ((uint64_t)(2 * t) * p) % (uint64_t)N) % (uint64_t)N);
    const int sA1 = (int)(((uint64_t)N - ((uint64_t)(2 * t + 1) * p) % (uint64_t)N) % (uint64_t)N);
    const double wA0 = exp2((double)sA0 / (double)N), wA1 = exp2((double)sA1 / (double)N);
    const double iwA0 = exp2(-(double)sA0 / (double)N), iwA1 = exp2(-(double)sA1 / (double)N);
    // kind of the two digits of column c, fixed for the whole test, 4 bits per column: bit 0 / 1:
    // digit 2m / 2m+1 has q + 1 bits; bit 2 / 3: its weight wrapped past N
    uint32_t kinds[(CA + 7) / 8];
#pragma unroll
    for (int w = 0; w < (CA + 7) / 8; ++w) kinds[w] = 0u;
#pragma unroll
    for (int c = 0; c < CA; ++c) {
        const int sb = sB[c];
        const bool o0 = sA0 + sb >= N, o1 = sA1 + sb >= N;
        const int s0 = o0 ? sA0 + sb - N : sA0 + sb;
        const int s1 = o1 ? sA1 + sb - N : sA1 + sb;
        const uint32_t kd = (uint32_t)(s0 < rem) | ((uint32_t)(s1 < rem) << 1) | ((uint32_t)o0 << 2) | ((uint32_t)o1 << 3);
        kinds[c / 8] |= kd << (4 * (c % 8));
    }
    auto kind = [&](int c) { return kinds[c / 8] >> (4 * (c % 8)); };
    // made opaque before each use: the weights and digit sizes derived from the kinds are then
    // formed where used, not hoisted into registers held across the transforms
    auto refresh_kinds = [&]() {
#pragma unroll
        for (int w = 0; w < (CA + 7) / 8; ++w) asm volatile("" : "+r"(kinds[w]));
    };

    // the digits between squarings: s_0 = 4 (digit 0 has weight 1)
    int x0s[CA], x1s[CA];
#pragma unroll
    for (int c = 0; c < CA; ++c) x0s[c] = x1s[c] = 0;
    if (t == 0) x0s[0] = 4;

    const NamedSync gsync{1u + (unsigned)seg, (unsigned)TL};
    double2* mybuf = bufs + seg * PADL;
    double maxerr = 0.0;
    uint64_t it = 0;
    uint32_t status = LLG_ST_OK;

    for (;;) {
        // ---- weight, radix-R0 DFT of the thread's two columns n, twiddle w_M^{n k0}, to segment
        //      order (one column's R0 values live at a time) ----
        refresh_kinds();
        if (holds) {
#pragma unroll
            for (int i = 0; i < NPT; ++i) {
                const int n = t + TA * i;
                double2 z[R0];
#pragma unroll
                for (int r = 0; r < R0; ++r) {
                    const int c = i + NPT * r;
                    const uint32_t kd = kind(c);
                    const double w = wB[c];
                    z[r] = make_double2(i2d_shift(x0s[c]) * (wA0 * w) * ((kd & 4u) ? 0.5 : 1.0),
                                        i2d_shift(x1s[c]) * (wA1 * w) * ((kd & 8u) ? 0.5 : 1.0));
                }
                dft_r0<R0>(z, omf);
                bufs[phys(n)] = z[0];
#pragma unroll
                for (int k0 = 1; k0 < R0; ++k0)
                    bufs[k0 * PADL + phys(n)] = cmul(z[k0], twiddle_m<M>(qtwM, (uint32_t)(n * k0), false));
            }
        }
        __syncthreads();
        double2 v[E];
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = mybuf[phys(tl + TL * i)];
        // the first pass stores after a segment barrier: the segment's loads above must be done
        radix_pass<GL, 0, false, true, NamedSync>(v, mybuf, qtwL, tl, gsync);
        gsync();
        forward_from<GL, 1>(v, mybuf, qtwL, tl, gsync);

        // ---- pair (k, M - k): real-FFT split + square (result scaled by 4, folded into iwB) ----
#pragma unroll
        for (int j = 0; j < E; ++j) mybuf[phys(tl * E + j)] = v[j];
        __syncthreads();
        {
            constexpr int RL = GL::RLAST, NB = E / RL;
            double2 wk[NB];
#pragma unroll
            for (int h = 0; h < NB; ++h)
                wk[h] = twiddle_m<M>(qtwM, (uint32_t)(R0 * freq_rev<GL>(tl * NB + h) + seg), false);
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const double2 A = v[j], Bc = conj2(bufs[pslot[j * T + t]]);  // conj(U_{M-k})
                const double2 s = cadd(A, Bc), d = csub(A, Bc);
                const double2 a3 = make_double2(3.0 * A.x - Bc.x, 3.0 * A.y - Bc.y);
                const double2 d2 = make_double2((d.x - d.y) * (d.x + d.y), 2.0 * d.x * d.y);
                v[j] = csub(cmul(a3, s), cmul(wk[j / RL], rot_k<RL, false>(d2, j % RL)));
            }
        }
        __syncthreads();  // partner reads (other segments) done before any segment stores
        inverse_from<GL, GL::P - 1, false>(v, mybuf, qtwL, tl, gsync);
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = cmul(v[i], twiddle_m<M>(qtwM, (uint32_t)((tl + TL * i) * seg), true));
        gsync();  // this segment's last inverse pass read its buffer
#pragma unroll
        for (int i = 0; i < E; ++i) mybuf[phys(tl + TL * i)] = v[i];
        __syncthreads();

        // ---- inverse radix-R0 DFT back to the thread's columns, then unweight, round and carry
        //      each column (the columns' carries are independent until the exchange below) ----
        double lerr = 0.0;
        refresh_kinds();
        if (holds) {
#pragma unroll
            for (int i = 0; i < NPT; ++i) {
                const int n = t + TA * i;
                double2 z[R0];
#pragma unroll
                for (int k0 = 0; k0 < R0; ++k0) z[k0] = bufs[k0 * PADL + phys(n)];
                dft_r0<R0>(z, omi);
#pragma unroll
                for (int r = 0; r < R0; ++r) {
                const int c = i + NPT * r;
                const uint32_t kd = kind(c);
                const double iw = iwB[c];
                const double a = z[r].x * (iwA0 * iw) * ((kd & 4u) ? 2.0 : 1.0);
                const double b = z[r].y * (iwA1 * iw) * ((kd & 8u) ? 2.0 : 1.0);
                long long la, lb;
                const double ra = round_shift(a, la), rb = round_shift(b, lb);
                lerr = fmax(lerr, fmax(fabs(a - ra), fabs(b - rb)));
                const int b0 = q + (int)(kd & 1u), b1 = q + (int)((kd >> 1) & 1u);  // digit sizes
                double cy;
                double x0 = dsplit_e(ra, b0, cy);
                const double x1 = dsplit_e(rb + cy, b1, cy);
                const double cout = cy;
                if (lane == 31) cbuf[warp * CA + c] = cout;
                const double cin = __shfl_up_sync(0xffffffffu, cout, 1);
                if (lane != 0) {
                    x0 = dsplit_e(x0 + cin, b0, cy);
                    x1s[c] = d2i_exact(x1 + cy);
                } else {
                    x1s[c] = d2i_exact(x1);
                }
                x0s[c] = d2i_exact(x0);
                }
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
        if (holds && lane == 0) {
#pragma unroll
            for (int c = 0; c < CA; ++c) {
                // m - 1 of m = t + TA c: the previous warp's last lane, or the last warp's last lane
                // of column c - 1 (column CA - 1 at m = 0: the wrap-around, 2^p == 1)
                double cin = (warp > 0) ? cbuf[(warp - 1) * CA + c] : cbuf[(WA - 1) * CA + ((c + CA - 1) % CA)];
                if (t == 0 && c == 0) cin -= 2.0;  // the "- 2" of s^2 - 2
                double cy;
                x0s[c] = d2i_exact(dsplit_e((double)x0s[c] + cin, q + (int)(kind(c) & 1u), cy));
                x1s[c] += (int)cy;
            }
        }
        ++it;
        if (bad) {
            status = LLG_ST_ROUNDOFF;
            break;
        }
        if (it >= iters) break;
    }

    if (holds && digits_out) {
        int64_t* out = digits_out + (size_t)blockIdx.x * N;
#pragma unroll
        for (int c = 0; c < CA; ++c) {
            const uint64_t m = (uint64_t)t + (uint64_t)TA * c;
            out[2 * m] = x0s[c];
            out[2 * m + 1] = x1s[c];
        }
    }
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

template <int R0, int LOG_L>
static size_t mixed_r_smem_bytes() {
    using MG = MixedRGeom<R0, LOG_L>;
    return sizeof(double2) * ((size_t)R0 * MG::PADL + MG::QLL + MG::QLM + 2 * R0 * R0) +
           sizeof(double) * (2 * MG::CA + MG::WA * MG::CA) + sizeof(int) * MG::CA + 2 * sizeof(unsigned long long) +
           sizeof(unsigned short) * MG::E * MG::T;  // partner slots of the real-FFT split
}

template <int R0, int LOG_L>
static cudaError_t launch_mixed_r_t(const SmallJob* jobs, int njobs, const double2* qtwL, const double2* qtwM,
                                    int64_t* digits, SmallResult* results, float* errlog, double abort_err,
                                    cudaStream_t st) {
    const size_t smem = mixed_r_smem_bytes<R0, LOG_L>();
    static PerDeviceOnce configured;
    if (!configured.done()) {
        cudaError_t e = cudaFuncSetAttribute(ll_small_fp64_mixed_r<R0, LOG_L>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured.mark();
    }
    ll_small_fp64_mixed_r<R0, LOG_L><<<njobs, MixedRGeom<R0, LOG_L>::T, smem, st>>>(jobs, qtwL, qtwM, digits,
                                                                                   results, errlog, abort_err);
    return cudaGetLastError();
}

template <int R0, int LOG_L>
static size_t mixed_smem_bytes() {
    using MG = MixedGeom<R0, LOG_L>;
    return sizeof(double2) * ((size_t)R0 * MG::PADL + MG::QLL + MG::QLM + 2 * R0 * R0) +
           sizeof(double) * (2 * MG::E + MG::W * MG::E) + sizeof(int) * MG::E + 2 * sizeof(unsigned long long);
}

template <int R0, int LOG_L>
static cudaError_t launch_mixed_t(const SmallJob* jobs, int njobs, const double2* qtwL, const double2* qtwM,
                                  int64_t* digits, SmallResult* results, float* errlog, double abort_err,
                                  cudaStream_t st) {
    const size_t smem = mixed_smem_bytes<R0, LOG_L>();
    static PerDeviceOnce configured;
    if (!configured.done()) {
        cudaError_t e = cudaFuncSetAttribute(ll_small_fp64_mixed<R0, LOG_L>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured.mark();
    }
    ll_small_fp64_mixed<R0, LOG_L><<<njobs, MixedGeom<R0, LOG_L>::T, smem, st>>>(jobs, qtwL, qtwM, digits,
                                                                                results, errlog, abort_err);
    return cudaGetLastError();
}

bool mixed_length_supported(uint32_t n, int* r0, int* log_l) {
    for (int r = 3; r <= 5; r += 2)
        for (int l = 9; l <= (r == 3 ? 11 : 10); ++l)
            if (n == 2u * (uint32_t)r << l) {
                if (r0) *r0 = r;
                if (log_l) *log_l = l;
                return true;
            }
    return false;
}

cudaError_t launch_small_fp64_mixed(uint32_t n, const SmallJob* jobs, int njobs, const double2* qtwL,
                                    const double2* qtwM, int64_t* digits, SmallResult* results,
                                    float* errlog, double abort_err, cudaStream_t st) {
    int r0 = 0, l = 0;
    if (!mixed_length_supported(n, &r0, &l)) return cudaErrorInvalidValue;
    if (r0 == 3) {
        switch (l) {
            case 9: return launch_mixed_r_t<3, 9>(jobs, njobs, qtwL, qtwM, digits, results, errlog, abort_err, st);
            case 10: return launch_mixed_r_t<3, 10>(jobs, njobs, qtwL, qtwM, digits, results, errlog, abort_err, st);
            case 11: return launch_mixed_t<3, 11>(jobs, njobs, qtwL, qtwM, digits, results, errlog, abort_err, st);
        }
    } else {
        switch (l) {
            case 9: return launch_mixed_r_t<5, 9>(jobs, njobs, qtwL, qtwM, digits, results, errlog, abort_err, st);
            case 10: return launch_mixed_t<5, 10>(jobs, njobs, qtwL, qtwM, digits, results, errlog, abort_err, st);
        }
    }
    return cudaErrorInvalidValue;
}

}  // namespace llg
