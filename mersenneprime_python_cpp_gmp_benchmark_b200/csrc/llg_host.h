// Host-side objects of the two-pass engine (internal; not part of the public ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "llg_internal.h"

namespace llg {

constexpr int kGraphChunk = 64;  // squarings per captured CUDA graph

bool large_length_supported(int log_n);
// N = R0 2^k two-pass lengths (R0 = 3, 5; k = 18 .. 21): R0 and the log2 row length they use.
bool large_mixed_length_supported(uint64_t n, int* r0, int* log_c);
int large_default_log_c(int log_n);
bool large_split_supported(int log_n, int log_c, int rows);
int set_error(int code, const char* msg);  // records this thread's llg_last_error() text
cudaError_t configure_large(int log_c, int g, int log_r);
cudaError_t seed_digits_device(int* digits, uint64_t n, cudaStream_t st);  // s_0 = 4, on the device
// Quarter-wave table of an L-point FFT in the padded layout the kernels read (entry r at qpad(r)).
std::vector<double2> padded_quarter_table(uint64_t L);
// Value of slot i of that layout (zero in the padding slots).
double2 padded_quarter_slot(uint64_t L, uint64_t i);
// The same quarter-wave table in the spread layout (entry r at qpad_s(r)).
std::vector<double2> spread_quarter_table(uint64_t L);

struct LargeTest {
    uint64_t p = 0, N = 0, M = 0;
    // logN: log2 N (-1 for N = R0 2^k); logR: large_col_code of the column length R
    int logN = 0, logC = 0, logR = 0, C = 0, R = 0, rows = 0, nblocks = 0, r0 = 1;
    double2* V = nullptr;
    double* carry = nullptr;
    double* carry2 = nullptr;
    LargeCtl* ctl = nullptr;
    unsigned* flags = nullptr;
    int* digits = nullptr;
    float* errlog = nullptr;
    int errlog_len = 0;
    double2 *qtwC = nullptr, *qtwR = nullptr, *qtwL = nullptr, *tw1 = nullptr, *tw2 = nullptr;
    int* pos_of_c = nullptr;
    double *wA = nullptr, *iwA = nullptr, *wB = nullptr, *iwB = nullptr;
    int *sA = nullptr, *sB = nullptr;
    LargeArgs args{};
    cudaGraphExec_t exec = nullptr;
    uint64_t done = 0;  // squarings enqueued since start()

    ~LargeTest();
    // n: the transform length (2^14 .. 2^23, or R0 2^k as large_mixed_length_supported); log_c < 0:
    // the default split; rows == 0: the default rows per row-pass block (power-of-two lengths)
    cudaError_t init(uint64_t p, uint64_t n, int log_c = -1, int rows = 0);
    cudaError_t start_seed(cudaStream_t st);    // s_0 = 4 written on the device, INIT + first squaring
    cudaError_t start_device(cudaStream_t st);  // the same from the digits already in `digits`
    cudaError_t step(uint64_t k, cudaStream_t st);                        // k more squarings
    cudaError_t step_plain(uint64_t k, bool dump_last, cudaStream_t st);
    cudaError_t final_pass(cudaStream_t st);                              // FINAL: digits on device
    cudaError_t finish(cudaStream_t st, std::vector<int>& out);           // FINAL: digits to host
    cudaError_t read_ctl(LargeCtl& h, cudaStream_t st);
    cudaError_t clear_err_since(cudaStream_t st);
    // k squarings, one launch at a time with events between the passes: mean device us per pass
    cudaError_t time_passes(uint64_t k, cudaStream_t st, double& row_us, double& col_us);
    // Diagnostic: one row pass with the wrap-around job withheld and waits bounded by spin_limit
    // sleeps, so tile 0 and the last tile give up; timed_out reports ctl->timeout. The state is
    // invalid afterwards.
    cudaError_t diag_withhold_wrap(unsigned long long spin_limit, cudaStream_t st, bool& timed_out);
};

// Device state of one exponent on the two-pass NTT engine (same launch sequence as LargeTest).
struct NttLargeTest {
    uint64_t p = 0, N = 0;
    int logN = 0, logC = 0, logR = 0, C = 0, R = 0, nblocks = 0;
    void* mem[20] = {};
    int nmem = 0;
    NttLargeArgs args{};
    cudaGraphExec_t exec = nullptr;
    uint64_t done = 0;
    LargeCtl* ctl = nullptr;
    int* digits = nullptr;

    ~NttLargeTest();
    cudaError_t init(uint64_t p, int log_n);
    cudaError_t start_seed(cudaStream_t st);
    cudaError_t start_device(cudaStream_t st);
    cudaError_t step(uint64_t k, cudaStream_t st);
    cudaError_t final_pass(cudaStream_t st);
    cudaError_t finish(cudaStream_t st, std::vector<int>& out);
    cudaError_t read_ctl(LargeCtl& h, cudaStream_t st);
    cudaError_t time_passes(uint64_t k, cudaStream_t st, double& row_us, double& col_us);
};

bool ntt_large_length_supported(int log_n);
// exact N-th root of 2, its inverse, w_N and N^-1 in GF(q) (host arithmetic)
bool ntt_host_constants(int log_n, uint64_t& omega, uint64_t& root2, uint64_t& inv_root2, uint64_t& invN);

}  // namespace llg
