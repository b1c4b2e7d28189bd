// Exact residue rebuild from signed variable-base digits, on the host, without GMP.
//
//   s = sum_j d_j * 2^ceil(jp/n)  mod  2^p - 1,  result in [0, 2^p - 1)
//
// This is the arithmetic of the reference's final-residue rebuild (lucaslehmer.cpp:312-323,
// cuda/ll_ntt.cu:238-252), which uses GMP; here it is a single carry sweep over the digits in
// bit order (digit j occupies bits [ceil(jp/n), ceil((j+1)p/n)) ), followed by folding the
// signed carry out of bit p back into bit 0 (2^p == 1 mod 2^p - 1) until it vanishes.
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/llgpu.h"

namespace {

typedef __int128 i128;
typedef unsigned __int128 u128;

inline uint64_t ceil_jp(uint64_t j, uint64_t p, uint64_t n) {
    return (uint64_t)(((u128)j * p + n - 1) / n);
}

// w: nw + 1 limbs, two's complement. Adds the signed value c at bit 0.
void add_signed(std::vector<uint64_t>& w, i128 c) {
    const uint64_t ext = (c < 0) ? ~0ull : 0ull;
    u128 acc = 0;
    uint64_t lo = (uint64_t)c, hi = (uint64_t)((u128)c >> 64);
    for (size_t i = 0; i < w.size(); ++i) {
        const uint64_t add = (i == 0) ? lo : (i == 1) ? hi : ext;
        acc = (u128)w[i] + add + (uint64_t)acc;
        w[i] = (uint64_t)acc;
        acc >>= 64;
    }
}

// Signed value of bits >= p (assumed small), and clears them.
i128 take_high(std::vector<uint64_t>& w, uint64_t p) {
    const size_t top = w.size() - 1;
    const bool neg = (w[top] >> 63) != 0;
    const size_t wi = p / 64;
    const unsigned off = (unsigned)(p % 64);
    // bits [p, p + 128) as a signed 128-bit value
    u128 lowpart = 0;
    {
        const uint64_t w0 = wi < w.size() ? w[wi] : (neg ? ~0ull : 0ull);
        const uint64_t w1 = wi + 1 < w.size() ? w[wi + 1] : (neg ? ~0ull : 0ull);
        const uint64_t w2 = wi + 2 < w.size() ? w[wi + 2] : (neg ? ~0ull : 0ull);
        lowpart = ((u128)w1 << 64) | w0;
        lowpart >>= off;
        if (off) lowpart |= ((u128)w2 << (128 - off));
    }
    const i128 high = (i128)lowpart;
    // clear bits >= p
    if (off) {
        w[wi] &= (1ull << off) - 1ull;
        for (size_t i = wi + 1; i < w.size(); ++i) w[i] = 0;
    } else {
        for (size_t i = wi; i < w.size(); ++i) w[i] = 0;
    }
    return high;
}

}  // namespace

extern "C" int llg_residue_from_digits(uint64_t p, uint32_t n, const int64_t* digits,
                                       uint64_t* words, size_t nwords, uint64_t* res64,
                                       int32_t* is_zero) {
    if (!digits || n == 0 || p < 2) return LLG_E_ARG;
    const size_t nw = (size_t)((p + 63) / 64);
    if (words && nwords < nw) return LLG_E_ARG;
    std::vector<uint64_t> w(nw + 3, 0);
    i128 carry = 0;
    uint64_t pos = 0;
    for (uint64_t j = 0; j < n; ++j) {
        const uint64_t next = ceil_jp(j + 1, p, n);
        const unsigned b = (unsigned)(next - pos);
        const i128 v = (i128)digits[j] + carry;
        if (b == 0) {
            carry = v;
            continue;
        }
        if (b > 62) return LLG_E_UNSUPPORTED;
        const uint64_t mask = (1ull << b) - 1ull;
        const uint64_t low = (uint64_t)v & mask;  // two's complement low bits = v mod 2^b
        carry = (v - (i128)low) >> b;             // exact floor division
        const size_t wi = pos / 64;
        const unsigned off = (unsigned)(pos % 64);
        w[wi] |= low << off;
        if (off + b > 64) w[wi + 1] |= low >> (64 - off);
        pos = next;
    }
    // value = w (p bits) + carry * 2^p  ==  w + carry  (mod 2^p - 1)
    for (int guard = 0; carry != 0 && guard < 1000; ++guard) {
        add_signed(w, carry);
        carry = take_high(w, p);
    }
    // canonical form: 2^p - 1 == 0
    bool all_ones = true;
    for (size_t i = 0; i < nw && all_ones; ++i) {
        const unsigned bits = (i + 1 < nw || p % 64 == 0) ? 64u : (unsigned)(p % 64);
        const uint64_t full = bits == 64 ? ~0ull : ((1ull << bits) - 1ull);
        if (w[i] != full) all_ones = false;
    }
    if (all_ones) std::fill(w.begin(), w.end(), 0ull);
    bool zero = true;
    for (size_t i = 0; i < nw; ++i)
        if (w[i]) zero = false;
    if (words) {
        std::memcpy(words, w.data(), nw * sizeof(uint64_t));
        for (size_t i = nw; i < nwords; ++i) words[i] = 0;
    }
    if (res64) *res64 = w[0];
    if (is_zero) *is_zero = zero ? 1 : 0;
    return LLG_OK;
}
