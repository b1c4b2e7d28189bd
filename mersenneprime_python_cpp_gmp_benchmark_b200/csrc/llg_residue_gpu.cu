// Exact residue rebuild on the GPU from device digits: s = sum_j d_j 2^ceil(jp/n) mod 2^p - 1,
// the arithmetic of the reference's final rebuild (lucaslehmer.cpp:312-323, cuda/ll_ntt.cu:238-252,
// done there with GMP on the host) and of the host-side llg_residue_from_digits, without copying
// the n digits back. The p-bit result is formed word by word:
//   1. every 64-bit word w takes the digits that start inside it, summed with their shifts as a
//      signed 128-bit S_w; T_w = low64(S_w) + (S_{w-1} >> 64) then has a carry-out e_w in
//      {-1, 0, 1} over the word's low 64 bits U_w (the carry of S_{w-1} is small);
//   2. the chains of +-1 carries through all-ones / all-zeros words are resolved by a scan of
//      per-chunk carry maps ({-1,0,1} -> {-1,0,1}, composed in one block);
//   3. the bits at and above p fold back into bit 0 (2^p == 1), by one thread with early exit;
//   4. 2^p - 1 (all ones) is the canonical zero.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/llgpu.h"

namespace llg {

namespace {

constexpr int kChunk = 64;  // words per chunk of the carry scan

__device__ __forceinline__ uint64_t off_of(uint64_t j, uint64_t p, uint64_t n) { return (j * p + n - 1) / n; }

// first digit starting at or after bit 64 w
__device__ __forceinline__ uint64_t first_digit(uint64_t w, uint64_t p, uint64_t n) {
    return w == 0 ? 0 : ((64 * w - 1) * n) / p + 1;
}

__device__ __int128 word_sum(uint64_t w, const int32_t* __restrict__ d, uint64_t p, uint64_t n) {
    uint64_t j0 = first_digit(w, p, n), j1 = first_digit(w + 1, p, n);
    if (j0 > n) j0 = n;
    if (j1 > n) j1 = n;
    __int128 s = 0;
    for (uint64_t j = j0; j < j1; ++j) s += (__int128)d[j] << (off_of(j, p, n) - 64 * w);
    return s;
}

// U_w and the carry-out e_w of T_w = low64(S_w) + (S_{w-1} >> 64); the top word also records
// S_{nw-1} >> 64 (what reaches past word nw - 1 before the +-1 chains)
__global__ void words_kernel(const int32_t* __restrict__ d, uint64_t p, uint64_t n, uint64_t nw,
                             uint64_t* __restrict__ U, int8_t* __restrict__ e, long long* top) {
    const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nw) return;
    const __int128 s = word_sum(w, d, p, n);
    const __int128 cin = (w > 0) ? (word_sum(w - 1, d, p, n) >> 64) : (__int128)0;
    const __int128 t = (__int128)(unsigned __int128)(uint64_t)s + cin;
    U[w] = (uint64_t)t;
    e[w] = (int8_t)(t >> 64);
    if (w == nw - 1) *top = (long long)(s >> 64);
}

// carry-out of one word for a carry-in x in {-1, 0, 1}
__device__ __forceinline__ int word_carry(uint64_t u, int e, int x) {
    int g = 0;
    if (x == 1 && u == ~0ull) g = 1;
    if (x == -1 && u == 0ull) g = -1;
    return e + g;
}

// map of chunk c: carry-in x -> carry-out, packed as three 2-bit fields (value + 1) for x = -1, 0, 1
__global__ void chunk_maps(const uint64_t* __restrict__ U, const int8_t* __restrict__ e, uint64_t nw,
                           uint8_t* __restrict__ maps, uint64_t nc) {
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const uint64_t w0 = c * kChunk, w1 = (w0 + kChunk < nw) ? w0 + kChunk : nw;
    int out[3];
    for (int k = 0; k < 3; ++k) {
        int x = k - 1;
        for (uint64_t w = w0; w < w1; ++w) x = word_carry(U[w], e[w], x);
        out[k] = x;
    }
    maps[c] = (uint8_t)((out[0] + 1) | ((out[1] + 1) << 2) | ((out[2] + 1) << 4));
}

__device__ __forceinline__ int apply_map(uint8_t m, int x) { return (int)((m >> (2 * (x + 1))) & 3u) - 1; }

// g after f
__device__ __forceinline__ uint8_t compose(uint8_t f, uint8_t g) {
    uint8_t r = 0;
    for (int k = 0; k < 3; ++k) r |= (uint8_t)((apply_map(g, apply_map(f, k - 1)) + 1) << (2 * k));
    return r;
}

// one block: the carry into every chunk (carry into chunk 0 is 0), and the carry out of the top
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) scan_maps(const uint8_t* __restrict__ maps, uint64_t nc,
                                                          int8_t* __restrict__ cin, int* top_carry) {
    __shared__ uint8_t agg[kScanThreads];
    const int t = threadIdx.x;
    const uint64_t per = (nc + kScanThreads - 1) / kScanThreads;
    const uint64_t c0 = t * per, c1 = (c0 + per < nc) ? c0 + per : nc;
    uint8_t f = 0x24;  // identity: -1 -> -1, 0 -> 0, 1 -> 1 (fields 0, 1, 2)
    for (uint64_t c = c0; c < c1; ++c) f = compose(f, maps[c]);
    agg[t] = f;
    __syncthreads();
    // inclusive scan of the maps in thread order (Hillis-Steele)
    for (int s = 1; s < kScanThreads; s <<= 1) {
        const uint8_t mine = agg[t];
        const uint8_t left = (t >= s) ? agg[t - s] : (uint8_t)0x24;
        __syncthreads();
        agg[t] = compose(left, mine);
        __syncthreads();
    }
    int x = (t == 0) ? 0 : apply_map(agg[t - 1], 0);
    for (uint64_t c = c0; c < c1; ++c) {
        cin[c] = (int8_t)x;
        x = apply_map(maps[c], x);
    }
    if (t == kScanThreads - 1) *top_carry = apply_map(agg[t], 0);
}

__global__ void apply_chunks(const uint64_t* __restrict__ U, const int8_t* __restrict__ e,
                             const int8_t* __restrict__ cin, uint64_t nw, uint64_t nc, uint64_t* __restrict__ F) {
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const uint64_t w0 = c * kChunk, w1 = (w0 + kChunk < nw) ? w0 + kChunk : nw;
    int x = cin[c];
    for (uint64_t w = w0; w < w1; ++w) {
        const uint64_t u = U[w];
        F[w] = u + (uint64_t)(long long)x;
        x = word_carry(u, e[w], x);
    }
}

// Adds the signed value h (|h| < 2^126) at bit 0 of the nw-word number F, with early exit; returns
// the signed carry out of the top word (two's complement words, extension of h's sign).
__device__ long long add_low(uint64_t* F, uint64_t nw, __int128 h) {
    unsigned __int128 acc = 0;
    const uint64_t ext = (h < 0) ? ~0ull : 0ull;
    const uint64_t lo = (uint64_t)h, hi = (uint64_t)((unsigned __int128)h >> 64);
    for (uint64_t i = 0; i < nw; ++i) {
        const uint64_t add = (i == 0) ? lo : (i == 1) ? hi : ext;
        acc = (unsigned __int128)F[i] + add + (uint64_t)acc;
        F[i] = (uint64_t)acc;
        acc >>= 64;
        // past h's words, a carry of 1 with ext all-ones (or 0 with ext 0) changes nothing more
        if (i >= 1 && ((ext == 0 && (uint64_t)acc == 0) || (ext == ~0ull && (uint64_t)acc == 1))) return 0;
    }
    // the top word was reached: the carry out is acc plus what of h lies above the words (its high
    // word when there is one word, else its sign extension)
    const long long rest = (nw == 1) ? (long long)hi : (ext ? -1ll : 0ll);
    return (long long)(uint64_t)acc + rest;
}

// bits >= p as a signed value (plus `above` units of 2^(64 nw)), cleared from F
__device__ __int128 take_high(uint64_t* F, uint64_t nw, uint64_t p, long long above) {
    const unsigned r = (unsigned)(p % 64);
    if (r == 0) return (__int128)above;  // 64 nw == p
    const uint64_t top = F[nw - 1];
    F[nw - 1] = top & ((1ull << r) - 1ull);
    return (__int128)(top >> r) + ((__int128)above << (64 - r));
}

// one thread: fold everything at and above bit p back into bit 0 until nothing is left
__global__ void fold_kernel(uint64_t* F, uint64_t nw, uint64_t p, const long long* top, const int* top_carry,
                            int* status) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    __int128 h = take_high(F, nw, p, *top + *top_carry);
    for (int guard = 0; h != 0; ++guard) {
        if (guard > 8) {
            *status = 1;
            return;
        }
        const long long over = add_low(F, nw, h);
        h = take_high(F, nw, p, over);
    }
    *status = 0;
}

// flags[0]: stays 1 while every word is all ones within p bits; flags[1]: 1 if any word is nonzero
__global__ void check_kernel(const uint64_t* __restrict__ F, uint64_t nw, uint64_t p, unsigned* flags) {
    const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool ones = true, nonzero = false;
    if (w < nw) {
        const unsigned r = (unsigned)(p % 64);
        const uint64_t full = (w == nw - 1 && r) ? ((1ull << r) - 1ull) : ~0ull;
        ones = F[w] == full;
        nonzero = F[w] != 0;
    }
    if (!__all_sync(0xffffffffu, ones) && (threadIdx.x & 31) == 0) atomicAnd(&flags[0], 0u);
    if (__any_sync(0xffffffffu, nonzero) && (threadIdx.x & 31) == 0) atomicOr(&flags[1], 1u);
}

}  // namespace

}  // namespace llg

extern "C" int llg_residue_from_digits_device(uint64_t p, uint32_t n, const int32_t* d_digits,
                                              uint64_t* d_words, uint64_t* res64, int32_t* is_zero,
                                              void* stream) {
    using namespace llg;
    if (!d_digits || n == 0 || p < 3) return LLG_E_ARG;
    if ((p + n - 1) / n > 62) return LLG_E_UNSUPPORTED;
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t nw = (p + 63) / 64, nc = (nw + kChunk - 1) / kChunk;
    // scratch: U, F (unless the caller's words), e, maps, chunk carries, scalars
    const size_t bytes = 2 * nw * sizeof(uint64_t) + nw + 2 * nc + 64;
    unsigned char* mem = nullptr;
    if (cudaMallocAsync(&mem, bytes, st) != cudaSuccess) return LLG_E_NOMEM;
    uint64_t* U = reinterpret_cast<uint64_t*>(mem);
    uint64_t* F = d_words ? d_words : U + nw;
    int8_t* e = reinterpret_cast<int8_t*>(mem + 2 * nw * sizeof(uint64_t));
    uint8_t* maps = reinterpret_cast<uint8_t*>(e + nw);
    int8_t* cin = reinterpret_cast<int8_t*>(maps + nc);
    unsigned char* sc = reinterpret_cast<unsigned char*>(cin + nc);
    sc = reinterpret_cast<unsigned char*>(((uintptr_t)sc + 15) & ~(uintptr_t)15);
    long long* top = reinterpret_cast<long long*>(sc);
    int* top_carry = reinterpret_cast<int*>(sc + 8);
    int* status = reinterpret_cast<int*>(sc + 12);
    unsigned* flags = reinterpret_cast<unsigned*>(sc + 16);
    static const unsigned init_flags[2] = {1u, 0u};
    int rc = LLG_OK;
    const unsigned B = 256;
    words_kernel<<<(unsigned)((nw + B - 1) / B), B, 0, st>>>(d_digits, p, n, nw, U, e, top);
    chunk_maps<<<(unsigned)((nc + B - 1) / B), B, 0, st>>>(U, e, nw, maps, nc);
    scan_maps<<<1, kScanThreads, 0, st>>>(maps, nc, cin, top_carry);
    apply_chunks<<<(unsigned)((nc + B - 1) / B), B, 0, st>>>(U, e, cin, nw, nc, F);
    fold_kernel<<<1, 32, 0, st>>>(F, nw, p, top, top_carry, status);
    cudaMemcpyAsync(flags, init_flags, sizeof init_flags, cudaMemcpyHostToDevice, st);
    check_kernel<<<(unsigned)((nw + B - 1) / B), B, 0, st>>>(F, nw, p, flags);
    unsigned hflags[2] = {0, 0};
    int hstatus = 0;
    uint64_t w0 = 0;
    cudaMemcpyAsync(hflags, flags, sizeof hflags, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&hstatus, status, sizeof hstatus, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&w0, F, sizeof w0, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = LLG_E_CUDA;
    if (!rc && hstatus) rc = LLG_E_CUDA;  // the fold did not settle (not reachable for valid digits)
    if (!rc && hflags[0] && d_words && cudaMemsetAsync(d_words, 0, nw * sizeof(uint64_t), st) != cudaSuccess)
        rc = LLG_E_CUDA;
    if (!rc) {
        const bool zero = hflags[0] || !hflags[1];
        if (res64) *res64 = zero ? 0 : w0;
        if (is_zero) *is_zero = zero ? 1 : 0;
    }
    cudaFreeAsync(mem, st);
    if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = LLG_E_CUDA;
    return rc;
}
