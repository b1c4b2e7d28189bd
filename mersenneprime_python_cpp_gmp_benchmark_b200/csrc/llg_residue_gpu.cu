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
// The inverse direction, digits_from_words, forms the digits of a residue at any length on the
// GPU (a test resumed or moved to a longer transform from a residue).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/llgpu.h"
#include "llg_internal.h"

namespace llg {

namespace {

constexpr int kChunk = 64;  // words per chunk of the carry scan

__device__ __forceinline__ uint64_t off_of(uint64_t j, uint64_t p, uint64_t n) { return (j * p + n - 1) / n; }

// first digit starting at or after bit 64 w
__device__ __forceinline__ uint64_t first_digit(uint64_t w, uint64_t p, uint64_t n) {
    return w == 0 ? 0 : ((64 * w - 1) * n) / p + 1;
}

template <class D>
__device__ __int128 word_sum(uint64_t w, const D* __restrict__ d, uint64_t p, uint64_t n) {
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

// Bits [s, s + b) of the p-bit residue in `words` (b <= 62, s + b <= p).
__device__ __forceinline__ uint64_t residue_bits(const uint64_t* __restrict__ words, uint64_t s, int b) {
    const uint64_t w = s >> 6;
    const int sh = (int)(s & 63);
    unsigned __int128 x = words[w] >> sh;
    if (sh + b > 64) x |= (unsigned __int128)words[w + 1] << (64 - sh);
    return (uint64_t)x & ((1ull << b) - 1ull);
}

// Digit j of s at length n, within one of balanced: raw bits r_j = bits [ceil(jp/n), ceil((j+1)p/n))
// of s; x_j = r_j - 2^b_j [r_j >= 2^(b_j - 1)] + [r_{j-1} >= 2^(b_{j-1} - 1)] (j - 1 of digit 0 is
// digit n - 1: 2^p == 1). Every carry comes from one digit's own top bit, so no chain forms:
// sum_j x_j 2^ceil(jp/n) == s mod 2^p - 1 and |x_j| <= 2^(b_j - 1).
__global__ void digits_from_words_kernel(const uint64_t* __restrict__ words, uint64_t p, uint64_t n,
                                         int32_t* __restrict__ digits) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint64_t jm = (j == 0) ? n - 1 : j - 1;
    const uint64_t s0 = off_of(j, p, n), s1 = off_of(j + 1, p, n), sm = off_of(jm, p, n), sm1 = off_of(jm + 1, p, n);
    const int b = (int)(s1 - s0), bm = (int)(sm1 - sm);
    const long long r = (long long)residue_bits(words, s0, b);
    const long long rm = (long long)residue_bits(words, sm, bm);
    const long long hi = (r >> (b - 1)) & 1, him = (rm >> (bm - 1)) & 1;
    digits[j] = (int32_t)(r - (hi << b) + him);
}

// One block per exponent of a whole-test batch (digits: cnt x n int64, natural order; the batch's
// job list gives p): the same rebuild as the kernels above, every step inside the block with the
// p-bit number in shared memory. Words and their carry-outs; the +-1 chains by per-thread segment
// maps and a block scan; the fold above p by one thread; the all-ones / zero check. Out per
// exponent: res64, flags (bit 0: residue zero, bit 1: the fold did not settle) and, with words
// non-null, the ceil(p/64) words at word_off[i].
constexpr int kBatchThreads = 256;
__global__ void __launch_bounds__(kBatchThreads) rebuild_batch_kernel(
    const int64_t* __restrict__ digits, const SmallJob* __restrict__ jobs, uint32_t n, uint64_t* __restrict__ res64,
    int32_t* __restrict__ flags, uint64_t* __restrict__ words, const uint64_t* __restrict__ word_off, uint64_t nw_cap) {
    extern __shared__ uint64_t F[];  // nw_cap words, then nw_cap carry-outs (int8)
    int8_t* e = reinterpret_cast<int8_t*>(F + nw_cap);
    __shared__ uint8_t agg[kBatchThreads];
    __shared__ long long s_top;
    __shared__ int s_top_carry, s_status, s_ones, s_nonzero;
    const int t = threadIdx.x, i = blockIdx.x;
    const uint64_t p = jobs[i].p, nw = (p + 63) / 64;
    const int64_t* d = digits + (size_t)i * n;
    if (t == 0) {
        s_status = 0;
        s_ones = 1;
        s_nonzero = 0;
    }
    for (uint64_t w = t; w < nw; w += kBatchThreads) {
        const __int128 sw = word_sum(w, d, p, n);
        const __int128 cin = (w > 0) ? (word_sum(w - 1, d, p, n) >> 64) : (__int128)0;
        const __int128 tw = (__int128)(unsigned __int128)(uint64_t)sw + cin;
        F[w] = (uint64_t)tw;
        e[w] = (int8_t)(tw >> 64);
        if (w == nw - 1) s_top = (long long)(sw >> 64);
    }
    __syncthreads();
    // the +-1 chains: map of each thread's segment of words, inclusive scan, then the carries in
    const uint64_t per = (nw + kBatchThreads - 1) / kBatchThreads;
    const uint64_t w0 = t * per, w1 = (w0 + per < nw) ? w0 + per : nw;
    uint8_t f = 0x24;  // identity map
    for (uint64_t w = w0; w < w1; ++w) {
        uint8_t m = 0;
        for (int k = 0; k < 3; ++k) m |= (uint8_t)((word_carry(F[w], e[w], k - 1) + 1) << (2 * k));
        f = compose(f, m);
    }
    agg[t] = f;
    __syncthreads();
    for (int sh = 1; sh < kBatchThreads; sh <<= 1) {
        const uint8_t mine = agg[t];
        const uint8_t left = (t >= sh) ? agg[t - sh] : (uint8_t)0x24;
        __syncthreads();
        agg[t] = compose(left, mine);
        __syncthreads();
    }
    int x = (t == 0) ? 0 : apply_map(agg[t - 1], 0);
    for (uint64_t w = w0; w < w1; ++w) {
        const uint64_t u = F[w];
        const int xo = word_carry(u, e[w], x);
        F[w] = u + (uint64_t)(long long)x;
        x = xo;
    }
    if (t == kBatchThreads - 1) s_top_carry = apply_map(agg[t], 0);
    __syncthreads();
    if (t == 0) {  // fold everything at and above bit p into bit 0
        __int128 h = take_high(F, nw, p, s_top + s_top_carry);
        for (int guard = 0; h != 0; ++guard) {
            if (guard > 8) {
                s_status = 1;
                break;
            }
            const long long over = add_low(F, nw, h);
            h = take_high(F, nw, p, over);
        }
    }
    __syncthreads();
    const unsigned r = (unsigned)(p % 64);
    bool ones = true, nonzero = false;
    for (uint64_t w = t; w < nw; w += kBatchThreads) {
        const uint64_t full = (w == nw - 1 && r) ? ((1ull << r) - 1ull) : ~0ull;
        ones = ones && F[w] == full;
        nonzero = nonzero || F[w] != 0;
    }
    if (!ones) atomicAnd(&s_ones, 0);
    if (nonzero) atomicOr(&s_nonzero, 1);
    __syncthreads();
    const bool zero = s_ones || !s_nonzero;  // 2^p - 1 (all ones) is the canonical zero
    if (t == 0) {
        res64[i] = zero ? 0 : F[0];
        flags[i] = (zero ? 1 : 0) | (s_status ? 2 : 0);
    }
    if (words) {
        uint64_t* out = words + word_off[i];
        for (uint64_t w = t; w < nw; w += kBatchThreads) out[w] = zero ? 0 : F[w];
    }
}

}  // namespace

cudaError_t rebuild_batch(const int64_t* d_digits, const SmallJob* d_jobs, int cnt, uint32_t n, uint64_t pmax,
                          uint64_t* d_res64, int32_t* d_flags, uint64_t* d_words, const uint64_t* d_word_off,
                          cudaStream_t st) {
    if (cnt <= 0) return cudaSuccess;
    const uint64_t nw_cap = (pmax + 63) / 64;
    const size_t smem = nw_cap * (sizeof(uint64_t) + 1) + 16;
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static PerDeviceOnce configured;
    if (!configured.done()) {
        const cudaError_t e = cudaFuncSetAttribute(rebuild_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   200 * 1024);
        if (e != cudaSuccess) return e;
        configured.mark();
    }
    rebuild_batch_kernel<<<cnt, kBatchThreads, smem, st>>>(d_digits, d_jobs, n, d_res64, d_flags, d_words, d_word_off,
                                                           nw_cap);
    return cudaGetLastError();
}

cudaError_t digits_from_words(uint64_t p, uint64_t n, const uint64_t* d_words, int32_t* d_digits, cudaStream_t st) {
    if (n == 0 || p < n || (p + n - 1) / n > 30) return cudaErrorInvalidValue;
    const unsigned B = 256;
    digits_from_words_kernel<<<(unsigned)((n + B - 1) / B), B, 0, st>>>(d_words, p, n, d_digits);
    return cudaGetLastError();
}

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
    count_h2d(sizeof init_flags);
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
