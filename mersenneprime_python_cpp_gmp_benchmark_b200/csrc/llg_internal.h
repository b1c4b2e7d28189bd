// Internal declarations shared by the kernels and the C-ABI layer (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

namespace llg {

// Per-device record of a one-time kernel setup (cudaFuncSetAttribute applies to the current device
// only): done() for the current device, mark() after the setup succeeded there. Devices 0..63; the
// race between two first launches is benign (the setup is idempotent).
struct PerDeviceOnce {
    std::atomic<unsigned long long> bits{0};
    static int current() {
        int d = 0;
        return cudaGetDevice(&d) == cudaSuccess && d >= 0 && d < 64 ? d : -1;
    }
    bool done() const {
        const int d = current();
        return d >= 0 && ((bits.load() >> d) & 1ull);
    }
    void mark() {
        const int d = current();
        if (d >= 0) bits.fetch_or(1ull << d);
    }
};

enum : uint32_t {
    LLG_ST_OK = 0,
    LLG_ST_ROUNDOFF = 1,  // a round-off distance exceeded the abort threshold
};

struct SmallJob {
    uint64_t p;
    uint64_t iters;  // squarings to run (>= 1)
};

struct SmallResult {
    double max_err;
    uint64_t iters_done;
    uint64_t ns;  // device time of the test (%globaltimer)
    uint32_t status;
    uint32_t pad;
};

// Whether the whole-test FP64 kernel of length 2^log_n reads its twiddle table in the spread
// layout (spread_quarter_table) rather than the padded one (padded_quarter_table).
bool small_fp64_spread_table(int log_n);
// FP64 whole-test kernel, N = 2^log_n with 5 <= log_n <= 13. digits: njobs * N int64 (may be null).
cudaError_t launch_small_fp64(int log_n, const SmallJob* jobs, int njobs, const double2* qtw,
                              int64_t* digits, SmallResult* results, float* errlog,
                              double abort_err, cudaStream_t st);

// FP64 whole-test kernel for N = 2 R0 2^l (R0 = 3: l = 9..11; R0 = 5: l = 9..10); qtwL / qtwM:
// padded quarter tables of 2^l and N/2 points.
bool mixed_length_supported(uint32_t n, int* r0, int* log_l);
cudaError_t launch_small_fp64_mixed(uint32_t n, const SmallJob* jobs, int njobs, const double2* qtwL,
                                    const double2* qtwM, int64_t* digits, SmallResult* results,
                                    float* errlog, double abort_err, cudaStream_t st);

// p < 256: exact multi-limb word arithmetic, one thread per exponent (4 limbs out per exponent).
cudaError_t launch_word(const SmallJob* jobs, int njobs, uint64_t* res, cudaStream_t st);

// Goldilocks constants of one NTT length N: an N-th root of 2, its inverse, N^-1 (mod q).
struct NttConst {
    uint64_t root2, inv_root2, invN;
};

// Exact NTT whole-test kernel, N = 2^log_n with 5 <= log_n <= 13 (qtw: padded half table of the
// N-point transform, gl::qpad8 layout).
cudaError_t launch_small_ntt(int log_n, const SmallJob* jobs, int njobs, const uint64_t* qtw, NttConst K,
                             int64_t* digits, SmallResult* results, cudaStream_t st);

// Adds `bytes` to the library's host-to-device copy count (llg_h2d_bytes).
void count_h2d(size_t bytes);

// Digits (int32, natural order, within one of balanced) at length n of the residue s in d_words
// (ceil(p/64) little-endian limbs, s < 2^p), formed on the GPU; enqueued on st. n <= p, digits of
// at most 30 bits.
cudaError_t digits_from_words(uint64_t p, uint64_t n, const uint64_t* d_words, int32_t* d_digits, cudaStream_t st);

// Exact residues of a whole-test batch on the GPU: cnt exponents (d_jobs[i].p <= pmax), n int64
// digits each (d_digits, natural order). Per exponent: d_res64[i], d_flags[i] (bit 0: residue zero,
// bit 1: failure) and, when d_words is non-null, the ceil(p/64) words at d_word_off[i]. Enqueued
// on st.
cudaError_t rebuild_batch(const int64_t* d_digits, const SmallJob* d_jobs, int cnt, uint32_t n, uint64_t pmax,
                          uint64_t* d_res64, int32_t* d_flags, uint64_t* d_words, const uint64_t* d_word_off,
                          cudaStream_t st);

// ---- two-pass engine (N = 2^16 .. 2^23): state resident in HBM ------------------------------

// Row-pass tiles of g rows of 2^log_c complex values that have kernels (LLG_ROW_SHAPES lists
// them as X(log_c, g)): g * 2^log_c / (values per thread) threads, a multiple of 32 up to 512,
// and at most ~180 KB of shared memory. large_rows_per_block is the default g of a row length.
#define LLG_ROW_SHAPES(X) \
    X(6, 4) X(6, 8) X(7, 2) X(7, 4) X(7, 8) X(8, 2) X(8, 4) X(8, 8) X(9, 2) X(9, 4) X(9, 8) X(10, 2) \
    X(10, 4) X(10, 8) X(11, 2) X(11, 4)
constexpr bool large_rows_supported(int log_c, int g) {
    return (log_c >= 6 && log_c <= 11) && (g == 2 || g == 4 || g == 8) && !(log_c == 6 && g == 2) &&
           !(log_c == 11 && g == 8);
}
#ifdef __CUDACC__
__host__ __device__
#endif
constexpr int large_rows_per_block(int log_c) { return log_c >= 11 ? 2 : 4; }
constexpr int kLargeLogE = 4;         // log2 of the complex values per thread in the column pass
constexpr unsigned long long kSpinLimit = 1ull << 22;  // x ~64 ns sleeps: ~0.3 s, then give up + flag
// log2 of the complex values per thread in the row pass of g rows of 2^log_c complex: 8 values
// (radix-8 passes, 64 registers a thread, two or more blocks per SM) for rows of up to 2^9, 16
// (radix-16 passes, 128 registers) for longer rows
#ifdef __CUDACC__
__host__ __device__
#endif
constexpr int large_row_log_e(int log_c, int g) { return (void)g, log_c <= 9 ? 3 : 4; }

struct LargeCtl {
    unsigned int epoch;              // squarings whose column pass has finished; +1 per column pass
    unsigned int ticket[2];          // row-pass block tickets, alternating by epoch parity
    unsigned int timeout;            // set when a bounded wait gave up (the result is then invalid)
    unsigned long long err_max;      // bits of the max round-off over the run (double, >= 0)
    unsigned long long err_since;    // same, since the host last cleared it
    unsigned int halo_read;          // NTT: epoch + 1 once block 0 has read the wrap-around rows
};

enum { LARGE_INIT = 0, LARGE_ITER = 1, LARGE_FINAL = 2 };

#ifdef __CUDACC__
// Bounded wait until *f >= target. On giving up it sets ctl->timeout (the run's result is then
// reported invalid) and returns, so a kernel never spins forever.
__device__ __forceinline__ void wait_flag(unsigned int* f, unsigned int target, LargeCtl* ctl,
                                          unsigned long long limit) {
    volatile unsigned int* vf = f;
    unsigned long long spins = 0;
    while (*vf < target) {
        if (++spins > limit) {
            atomicExch(&ctl->timeout, 1u);
            break;
        }
        __nanosleep(64);
    }
    __threadfence();
}
#endif

struct LargeArgs {
    double2* V;               // state: element (row a, column slot pos) at pos * R + a
    const double2* qtwC;      // full padded twiddle table of the C-point row FFT
    const double2* qtwR;      // quarter table of the R-point column FFT (spread layout for a
                              // power-of-two R, padded for R = R0 L)
    const double2* qtwL;      // R = R0 L: padded quarter table of the L-point column sub-FFTs
    const double2* tw1;       // e^{-2 pi i x / M}, x < 2^tw_shift
    const double2* tw2;       // e^{-2 pi i y 2^tw_shift / M}
    const int* pos_of_c;      // column slot of row-FFT frequency c
    const double* wA;         // [2R] 2^(sA/N) of digit 2a+e
    const double* iwA;        // [2R] 2^(-sA/N)
    const int* sA;            // [2R] (-(2a+e) p) mod N
    const double* wB;         // [C] 2^(sB/N)
    const double* iwB;        // [C] 2^(-sB/N) / (4M)
    const int* sB;            // [C] (-2Rb p) mod N
    double* carry;            // [nblocks + 1][C] hop-1 carry-outs of a tile's last row (integers):
                              // slot 0 the wrap-around job's (row R-1, one column on), k + 1 tile k's
    double* carry2;           // [nblocks + 1][C] hop-2 carry-outs (integers of a few units)
    LargeCtl* ctl;
    unsigned int* flags;      // [nblocks + 1] epoch + 1 once the job of that slot published its carries
    unsigned long long spin_limit;  // bound of every wait on a flag (x ~64 ns sleeps)
    int* digits;              // N int32, natural order (INIT input; dump / FINAL output)
    float* errlog;            // per-epoch max round-off ring (may be null)
    int errlog_len;
    int dump;                 // ITER: also write the digits
    int tw_shift;
    int C, R, nblocks;
    int q, rem;               // p / N, p % N
    int N;                    // transform length: 2^k, or 3 x 2^k / 5 x 2^k (R = R0 L)
    int logN;                 // log2 N for a power of two
};

// Row pass; grid > 0 overrides the block count (nblocks, + 1 for the wrap-around job unless INIT).
cudaError_t launch_large_row(int log_c, int g, int mode, const LargeArgs& a, cudaStream_t st, int grid = 0);
// Column-length code of the two-pass engine: log2 R for a power of two, 100 R0 + log2 L for the
// column length R = R0 L (launch_large_col and configure_large take it).
constexpr int large_col_code(int r0, int log_l) { return r0 == 1 ? log_l : 100 * r0 + log_l; }
cudaError_t launch_large_col(int log_r, const LargeArgs& a, cudaStream_t st);

// ---- two-pass exact NTT engine (N = 2^14 .. 2^23): N field elements in HBM ------------------

struct NttLargeArgs {
    uint64_t* V;              // state: element (row a, column slot pos) at pos * R + a
    const uint64_t* qtwC;     // padded half table of the C-point row NTT (gl::qpad8)
    const uint64_t* qtwR;     // padded half table of the R-point column NTT
    const uint64_t* tw1;      // w_N^x, x < 2^tw_shift
    const uint64_t* tw2;      // w_N^(y 2^tw_shift)
    const int* pos_of_c;      // column slot of row-NTT frequency c
    const uint64_t* wA;       // [R] w^sA(a), w an N-th root of 2
    const uint64_t* iwA;      // [R] w^-sA(a)
    const int* sA;            // [R] (-a p) mod N
    const uint64_t* wB;       // [C] w^sB(b)
    const uint64_t* iwB;      // [C] w^-sB(b) / N
    const int* sB;            // [C] (-R b p) mod N
    long long* c1;            // [nblocks][C] hop-1 carry-outs of each block's last row
    int* c2;                  // [nblocks][C] hop-2 carry-outs
    int* c3;                  // [nblocks][C] hop-3 carry-outs
    long long* halo;          // block 0's wrap-around carries: C int64 + 2 * C int32
    LargeCtl* ctl;
    unsigned int* flags;      // [nblocks] epoch + 1 once block k published its carries
    int* digits;              // N int32, natural order (INIT input; dump / FINAL output)
    int dump;
    int tw_shift;
    int C, R, nblocks;
    int q, rem;
    int logN;
};

cudaError_t launch_ntt_row(int log_c, int mode, const NttLargeArgs& a, cudaStream_t st);
cudaError_t launch_ntt_col(int log_r, const NttLargeArgs& a, cudaStream_t st);
cudaError_t configure_ntt_large(int log_c, int log_r);

}  // namespace llg
