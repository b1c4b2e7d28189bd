// Internal declarations shared by the kernels and the C-ABI layer (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace llg {

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

// FP64 whole-test kernel, N = 2^log_n with 5 <= log_n <= 13. digits: njobs * N int64 (may be null).
cudaError_t launch_small_fp64(int log_n, const SmallJob* jobs, int njobs, const double2* qtw,
                              int64_t* digits, SmallResult* results, float* errlog,
                              double abort_err, cudaStream_t st);

// p < 64: exact 128-bit word arithmetic, one thread per exponent.
cudaError_t launch_word(const SmallJob* jobs, int njobs, uint64_t* res, cudaStream_t st);

}  // namespace llg
