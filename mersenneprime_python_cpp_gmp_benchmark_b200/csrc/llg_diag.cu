// Peak-throughput probes used as roofline denominators (the driver-written peaks file has HBM
// bandwidth and tensor-core throughput only): dependent FP64 FMA chains and dependent 32-bit
// IMAD chains, 8 independent chains per thread, every SM filled.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/llgpu.h"

namespace {

__global__ void fp64_fma_probe(double* out, int iters, double b, double c) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = 1e-3 * (threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
    }
    double s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 123.456) out[0] = s;  // keeps the chains live; never true for these inputs
}

__global__ void int32_mad_probe(uint32_t* out, int iters, uint32_t b, uint32_t c) {
    uint32_t a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = threadIdx.x * 2654435761u + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = a[k] * b + c;
    }
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s ^= a[k];
    if (s == 0x12345678u) out[0] = s;
}

}  // namespace

// ops/s of the probe (FP64: 2 flops per FMA; INT32: 1 multiply-add per IMAD).
extern "C" int llg_measure_peak(int which, double* ops_per_s) {
    if (!ops_per_s) return LLG_E_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return LLG_E_NODEV;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    void* out = nullptr;
    if (cudaMalloc(&out, 64) != cudaSuccess) return LLG_E_NOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int threads = 256, blocks = sms * 8, iters = 1 << 14;
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        if (which == 0)
            fp64_fma_probe<<<blocks, threads>>>((double*)out, iters, 0.999999, 1e-7);
        else
            int32_mad_probe<<<blocks, threads>>>((uint32_t*)out, iters, 2654435761u, 12345u);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return LLG_E_CUDA;
    const double ops = (double)blocks * threads * iters * 8 * (which == 0 ? 2.0 : 1.0);
    *ops_per_s = ops / (best * 1e-3);
    return LLG_OK;
}
