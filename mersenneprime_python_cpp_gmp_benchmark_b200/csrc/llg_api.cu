// The C-ABI boundary (include/llgpu.h): engine selection, transform-length choice, per-thread
// CUDA streams and buffers, the round-off escalation loop and the exact residue rebuild.
// Everything numerical runs on the GPU; the host only sizes, launches, and turns digits into the
// residue (llg_residue.cpp). There is no CPU fallback: a CUDA failure is an error status.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/llgpu.h"
#include "llg_host.h"
#include "llg_device.cuh"
#include "llg_internal.h"

namespace {

// padded layout of the NTT quarter tables (same as gl::qpad8 in llg_ntt.cuh)
constexpr uint32_t gl_qpad8(uint32_t r) { return r + (r >> 4); }
constexpr uint32_t gl_qpad8_len(uint32_t qm) { return qm + (qm >> 4) + 1; }

using namespace llg;

thread_local std::string t_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return code;
}

#define CK(x)                                                                                 \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess)                                                                \
            return fail(e_ == cudaErrorMemoryAllocation ? LLG_E_NOMEM : LLG_E_CUDA,           \
                        "CUDA: %s at %s (%s:%d)", cudaGetErrorString(e_), #x, __FILE__, __LINE__); \
    } while (0)

double g_max_bpw = 18.0;  // lucaslehmer.cpp:246
std::mutex g_mx;
// Round-off bound: a test whose worst |x - round(x)| exceeds it is redone at a longer length (the
// reference's bound is 0.35 with a GMP redo, lucaslehmer.cpp:296; llg_set_roundoff_limit).
std::atomic<double> g_abort_err{0.4};

constexpr int kSmallLogMin = 5;   // N = 32
constexpr int kSmallLogMax = 13;  // N = 8192

// ---- device tables ------------------------------------------------------------------------

struct DeviceTables {
    std::map<uint32_t, double2*> qtw;      // quarter-wave twiddles of the M-point FFT, by M
    std::map<uint32_t, double2*> qtw_s;    // the same in the spread layout (qpad_s), by M
    uint64_t* nqtw[kSmallLogMax + 1] = {}; // NTT: padded quarter table of the N-point transform
    NttConst nk[kSmallLogMax + 1] = {};
};

// ---- Goldilocks arithmetic on the host (tables): cuda/ll_ntt.cu:42-44, 182-195 ---------------

constexpr uint64_t kGQ = 0xFFFFFFFF00000001ull;
uint64_t hmul(uint64_t a, uint64_t b) { return (uint64_t)(((unsigned __int128)a * b) % kGQ); }
uint64_t hpow(uint64_t a, uint64_t e) {
    uint64_t r = 1;
    a %= kGQ;
    while (e) {
        if (e & 1) r = hmul(r, a);
        a = hmul(a, a);
        e >>= 1;
    }
    return r;
}
uint64_t hinv(uint64_t a) { return hpow(a, kGQ - 2); }

// w_N = 7^((q-1)/N) and an N-th root of 2 from a primitive (192 N)-th root (2 has order 192)
bool ntt_constants(int log_n, uint64_t& omega, NttConst& K) {
    const uint64_t N = 1ull << log_n;
    omega = hpow(7, (kGQ - 1) / N);
    const uint64_t om = hpow(7, (kGQ - 1) / (192 * N)), r192 = hpow(om, N);
    uint64_t pw = 1, s = 0;
    for (; s < 192; ++s) {
        if (pw == 2) break;
        pw = hmul(pw, r192);
    }
    if (s == 192) return false;
    K.root2 = hpow(om, s);
    K.inv_root2 = hinv(K.root2);
    K.invN = hinv(N % kGQ);
    return true;
}
std::map<int, DeviceTables> g_tables;  // per device ordinal

void load_tuning_once(int dev);

int device_ready(int* dev_out) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(LLG_E_NODEV, "no CUDA device visible (%s)",
                    e != cudaSuccess ? cudaGetErrorString(e) : "device count 0");
    }
    CK(cudaGetDevice(dev_out));
    load_tuning_once(*dev_out);
    return LLG_OK;
}

int get_qtw(int dev, uint32_t m, const double2** out, bool spread = false) {
    std::lock_guard<std::mutex> lk(g_mx);
    DeviceTables& T = g_tables[dev];
    double2*& d = spread ? T.qtw_s[m] : T.qtw[m];
    if (!d) {
        // padded layout (qpad), or the spread one (qpad_s)
        std::vector<double2> h = spread ? spread_quarter_table(m) : padded_quarter_table(m);
        CK(cudaMalloc(&d, h.size() * sizeof(double2)));
        CK(cudaMemcpy(d, h.data(), h.size() * sizeof(double2), cudaMemcpyHostToDevice));
        count_h2d(h.size() * sizeof(double2));
    }
    *out = d;
    return LLG_OK;
}

int get_ntt(int dev, int log_n, const uint64_t** qtw, NttConst* K) {
    std::lock_guard<std::mutex> lk(g_mx);
    DeviceTables& T = g_tables[dev];
    if (!T.nqtw[log_n]) {
        uint64_t omega;
        NttConst k;
        if (!ntt_constants(log_n, omega, k)) return fail(LLG_E_UNSUPPORTED, "no N-th root of 2 for N=2^%d", log_n);
        const uint32_t QL = (1u << log_n) / 2;  // half table
        std::vector<uint64_t> h(gl_qpad8_len(QL), 0ull);
        uint64_t w = 1;
        for (uint32_t r = 0; r < QL; ++r) {
            h[gl_qpad8(r)] = w;
            w = hmul(w, omega);
        }
        uint64_t* d = nullptr;
        CK(cudaMalloc(&d, h.size() * sizeof(uint64_t)));
        CK(cudaMemcpy(d, h.data(), h.size() * sizeof(uint64_t), cudaMemcpyHostToDevice));
        count_h2d(h.size() * sizeof(uint64_t));
        T.nqtw[log_n] = d;
        T.nk[log_n] = k;
    }
    *qtw = T.nqtw[log_n];
    *K = T.nk[log_n];
    return LLG_OK;
}

// ---- lengths --------------------------------------------------------------------------------

int ilog2_exact(uint64_t n) {
    if (n == 0 || (n & (n - 1))) return -1;
    int l = 0;
    while ((1ull << l) < n) ++l;
    return l;
}

constexpr uint64_t kMaxDigitBits = 28;  // FP64 digits are held as int32 between iterations
constexpr uint64_t kWordMaxP = 256;     // p below this runs on the exact multi-limb word kernel

// A length is usable when every digit has enough bits for the one-exchange balanced carry to stay
// balanced (floor(p/N) >= log2(N)/2 + 2: the carry into a digit is ~sqrt(N) times smaller than its
// base) and few enough for int32 digits and FP64 products.
constexpr int kLargeLogMax = 23;

bool is_small_pow2_length(uint64_t n) {
    const int l = ilog2_exact(n);
    return l >= kSmallLogMin && l <= kSmallLogMax;
}

// lengths of the whole-test kernels: 2^5 .. 2^13 and 3 x 2^10, 5 x 2^10, 3 x 2^11, 5 x 2^11, 3 x 2^12
bool is_small_length(uint64_t n) {
    return is_small_pow2_length(n) || (n < (1ull << 32) && mixed_length_supported((uint32_t)n, nullptr, nullptr));
}

int ceil_log2(uint64_t n) {
    int l = 0;
    while ((1ull << l) < n) ++l;
    return l;
}

// every FP64 length, ascending
const std::vector<uint32_t>& fp64_lengths() {
    static const std::vector<uint32_t> v = [] {
        std::vector<uint32_t> a;
        for (int l = kSmallLogMin; l <= kLargeLogMax; ++l) a.push_back(1u << l);
        for (uint32_t n = 1024; n <= (1u << 14); ++n)
            if (mixed_length_supported(n, nullptr, nullptr)) a.push_back(n);
        for (uint32_t r = 3; r <= 5; r += 2)
            for (int k = 18; k <= 21; ++k)
                if (large_mixed_length_supported((uint64_t)r << k, nullptr, nullptr)) a.push_back(r << k);
        std::sort(a.begin(), a.end());
        return a;
    }();
    return v;
}

// The two-pass engine's three-hop carry keeps digits balanced down to ~log2(N)/4 + 1 bits per
// digit; it asks for floor(p/N) >= log2(N)/4 + 3.
// Two-pass FP64 lengths: 2^14 .. 2^23 and R0 2^k (large_mixed_length_supported).
bool large_fp64_length(uint64_t n) {
    const int l = ilog2_exact(n);
    return (l > kSmallLogMax && large_length_supported(l)) || large_mixed_length_supported(n, nullptr, nullptr);
}

bool fp64_length_usable(uint64_t p, uint64_t n) {
    if (n == 0 || (p + n - 1) / n > kMaxDigitBits) return false;
    if (is_small_length(n)) return 2 * (p / n) >= (uint64_t)ceil_log2(n) + 4;
    if (large_fp64_length(n)) return 4 * (p / n) >= (uint64_t)ceil_log2(n) + 12;
    return false;
}

// smallest usable length with p / N <= bpw
// Length choices of the autotuner (llg_set_length_choice): where the bits-per-digit rule gives a
// whole-test length N, use the recorded length instead (when usable for p). Indexed by N's
// position in fp64_lengths(); 0 = the rule's own length.
constexpr size_t kMaxLengths = 64;
std::atomic<uint32_t> g_length_choice[kMaxLengths];

int length_index(uint32_t n) {
    const std::vector<uint32_t>& v = fp64_lengths();
    for (size_t i = 0; i < v.size() && i < kMaxLengths; ++i)
        if (v[i] == n) return (int)i;
    return -1;
}

uint32_t fp64_length(uint64_t p, double bpw) {
    for (uint32_t N : fp64_lengths())
        if ((double)p / (double)N <= bpw && fp64_length_usable(p, N)) {
            const int i = length_index(N);
            const uint32_t c = i >= 0 ? g_length_choice[i].load() : 0u;
            return (c && fp64_length_usable(p, c)) ? c : N;
        }
    return 0;
}

// NTT: exact while every convolution output stays below q/2, i.e. ceil(p/N) <= (63 - log2 N)/2
// (cuda/ll_ntt.cu:172-175); the same bits-per-digit floor as the FP64 engines keeps the four-hop
// carry balanced.
constexpr int kNttLogMin = 6;  // N = 64, the reference's shortest NTT (cuda/ll_ntt.cu:177)

bool ntt_length_usable(uint64_t p, uint64_t n) {
    const int l = ilog2_exact(n);
    if (l < kNttLogMin || (l > kSmallLogMax && !ntt_large_length_supported(l))) return false;
    return (p + n - 1) / n <= (uint64_t)((63 - l) / 2) && 4 * (p / n) >= (uint64_t)l + 12;
}

uint32_t ntt_len(uint64_t p) {
    if (p < kWordMaxP) return 0;
    for (int l = kNttLogMin; l <= kLargeLogMax; ++l)
        if (ntt_length_usable(p, 1ull << l)) return 1u << l;
    return 0;
}

uint32_t next_fp64_length(uint64_t p, uint32_t n) {
    for (uint32_t N : fp64_lengths())
        if (N > n && fp64_length_usable(p, N)) return N;
    return 0;
}

// ---- batches: exponents grouped by length, one launch per group, groups on their own streams --

struct Item {
    size_t idx;  // position in the caller's arrays
    uint64_t p;
    uint64_t iters;
    uint32_t n;  // 0: word path (p < 64)
    uint32_t escalations;
};

struct Group {
    uint32_t n = 0;  // 0 = word path
    std::vector<Item> items;
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    void* d_jobs = nullptr;
    void* d_results = nullptr;  // SmallResult[] or uint64_t[] (word path)
    void* d_digits = nullptr;
    // the residues rebuilt on the device from d_digits: res64, flags (bit 0 zero), words (optional)
    uint64_t* d_res64 = nullptr;
    int32_t* d_rflags = nullptr;
    uint64_t* d_words = nullptr;
    uint64_t* d_word_off = nullptr;
    uint64_t pmax = 0;
    size_t total_words = 0;
};

void set_trivial(llg_result* r, uint64_t p) {
    std::memset(r, 0, sizeof *r);
    r->p = p;
    r->status = LLG_OK;
    r->is_zero = (p == 2) ? 1 : 0;  // lucaslehmer.cpp:31-33: p<2 and even p composite, p=2 prime
}

}  // namespace

struct llg_batch {
    int dev = -1;
    int engine = LLG_ENGINE_FP64;
    size_t count = 0;
    std::vector<uint64_t> ps;
    std::vector<llg_result> out;
    std::vector<Group> groups;
    std::vector<Item> large;      // two-pass engine exponents, run one at a time at collect
    cudaEvent_t fork = nullptr;   // recorded on the caller's stream at launch (timing enabled)
    cudaEvent_t joined = nullptr; // recorded on the caller's stream after every group joined
    bool launched = false;
    bool collected = false;
    bool keep_words = false;
    std::vector<std::vector<uint64_t>> words;  // per exponent, when keep_words
    float* d_errlog = nullptr;  // optional per-iteration round-off log (single-exponent batches)
    uint64_t errlog_len = 0;
};

namespace {

void release_group(Group& g) {
    if (g.st) {
        for (void* ptr : {g.d_jobs, g.d_results, g.d_digits, (void*)g.d_res64, (void*)g.d_rflags, (void*)g.d_words,
                          (void*)g.d_word_off})
            if (ptr) cudaFreeAsync(ptr, g.st);
        cudaStreamSynchronize(g.st);
        cudaStreamDestroy(g.st);
    }
    if (g.done) cudaEventDestroy(g.done);
    g = Group();
}

void destroy_batch(llg_batch* b) {
    if (!b) return;
    for (Group& g : b->groups) release_group(g);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->joined) cudaEventDestroy(b->joined);
    if (b->d_errlog) cudaFree(b->d_errlog);
    delete b;
}

// Allocates and uploads one group's job list (synchronously on the group's stream).
int setup_group(Group& g, bool keep_words) {
    CK(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
    const size_t cnt = g.items.size();
    // longest first: the block scheduler then hands out the tests in LPT order
    std::sort(g.items.begin(), g.items.end(), [](const Item& a, const Item& b) { return a.iters > b.iters; });
    std::vector<SmallJob> jobs(cnt);
    for (size_t i = 0; i < cnt; ++i) jobs[i] = SmallJob{g.items[i].p, g.items[i].iters};
    CK(cudaMallocAsync(&g.d_jobs, cnt * sizeof(SmallJob), g.st));
    if (g.n == 0) {
        CK(cudaMallocAsync(&g.d_results, cnt * 4 * sizeof(uint64_t), g.st));
    } else {
        CK(cudaMallocAsync(&g.d_results, cnt * sizeof(SmallResult), g.st));
        CK(cudaMallocAsync(&g.d_digits, cnt * (size_t)g.n * sizeof(int64_t), g.st));
        CK(cudaMallocAsync(&g.d_res64, cnt * sizeof(uint64_t), g.st));
        CK(cudaMallocAsync(&g.d_rflags, cnt * sizeof(int32_t), g.st));
        g.pmax = 0;
        for (const Item& it : g.items) g.pmax = std::max(g.pmax, it.p);
        if (keep_words) {
            std::vector<uint64_t> off(cnt);
            g.total_words = 0;
            for (size_t i = 0; i < cnt; ++i) {
                off[i] = g.total_words;
                g.total_words += (size_t)((g.items[i].p + 63) / 64);
            }
            CK(cudaMallocAsync(&g.d_words, g.total_words * sizeof(uint64_t), g.st));
            CK(cudaMallocAsync(&g.d_word_off, cnt * sizeof(uint64_t), g.st));
            CK(cudaMemcpyAsync(g.d_word_off, off.data(), cnt * sizeof(uint64_t), cudaMemcpyHostToDevice, g.st));
            count_h2d(cnt * sizeof(uint64_t));
        }
    }
    CK(cudaMemcpyAsync(g.d_jobs, jobs.data(), cnt * sizeof(SmallJob), cudaMemcpyHostToDevice, g.st));
    count_h2d(cnt * sizeof(SmallJob));
    CK(cudaStreamSynchronize(g.st));
    return LLG_OK;
}

int launch_group(llg_batch* b, Group& g, cudaStream_t caller) {
    CK(cudaStreamWaitEvent(g.st, b->fork, 0));
    const int cnt = (int)g.items.size();
    if (g.n == 0) {
        CK(launch_word((const SmallJob*)g.d_jobs, cnt, (uint64_t*)g.d_results, g.st));
    } else if (b->engine == LLG_ENGINE_NTT) {
        const uint64_t* qtw = nullptr;
        NttConst K;
        int rc = get_ntt(b->dev, ilog2_exact(g.n), &qtw, &K);
        if (rc) return rc;
        CK(launch_small_ntt(ilog2_exact(g.n), (const SmallJob*)g.d_jobs, cnt, qtw, K, (int64_t*)g.d_digits,
                            (SmallResult*)g.d_results, g.st));
    } else if (is_small_pow2_length(g.n)) {
        const double2* qtw = nullptr;
        int rc = get_qtw(b->dev, g.n / 2, &qtw, small_fp64_spread_table(ilog2_exact(g.n)));
        if (rc) return rc;
        float* elog = (cnt == 1) ? b->d_errlog : nullptr;
        CK(launch_small_fp64(ilog2_exact(g.n), (const SmallJob*)g.d_jobs, cnt, qtw, (int64_t*)g.d_digits,
                             (SmallResult*)g.d_results, elog, g_abort_err.load(), g.st));
    } else {
        int r0 = 0, ll = 0;
        mixed_length_supported(g.n, &r0, &ll);
        const double2 *qtwL = nullptr, *qtwM = nullptr;
        int rc = get_qtw(b->dev, 1u << ll, &qtwL);
        if (!rc) rc = get_qtw(b->dev, g.n / 2, &qtwM);
        if (rc) return rc;
        float* elog = (cnt == 1) ? b->d_errlog : nullptr;
        CK(launch_small_fp64_mixed(g.n, (const SmallJob*)g.d_jobs, cnt, qtwL, qtwM, (int64_t*)g.d_digits,
                                   (SmallResult*)g.d_results, elog, g_abort_err.load(), g.st));
    }
    if (g.n) {
        // exact residues on the device: only res64 and the zero flag (and words when kept) come back
        CK(rebuild_batch((const int64_t*)g.d_digits, (const SmallJob*)g.d_jobs, cnt, g.n, g.pmax, g.d_res64,
                         g.d_rflags, g.d_words, g.d_word_off, g.st));
    }
    CK(cudaEventRecord(g.done, g.st));
    CK(cudaStreamWaitEvent(caller, g.done, 0));
    return LLG_OK;
}

// Reads one finished group back; items that aborted on round-off go to `retry` at a longer length.
int collect_group(llg_batch* b, Group& g, std::vector<Item>& retry) {
    const size_t cnt = g.items.size();
    CK(cudaEventSynchronize(g.done));
    if (g.n == 0) {
        std::vector<uint64_t> res(cnt * 4);
        CK(cudaMemcpyAsync(res.data(), g.d_results, cnt * 4 * sizeof(uint64_t), cudaMemcpyDeviceToHost, g.st));
        CK(cudaStreamSynchronize(g.st));
        for (size_t i = 0; i < cnt; ++i) {
            llg_result& r = b->out[g.items[i].idx];
            const uint64_t* w = res.data() + 4 * i;
            const size_t nw = (size_t)((g.items[i].p + 63) / 64);
            if (b->keep_words) b->words[g.items[i].idx].assign(w, w + nw);
            r.iters = g.items[i].iters;
            r.res64 = w[0];
            r.is_zero = (w[0] | w[1] | w[2] | w[3]) == 0;
            r.n = 1;
            r.status = LLG_OK;
        }
        return LLG_OK;
    }
    const uint32_t n = g.n;
    std::vector<SmallResult> res(cnt);
    std::vector<uint64_t> r64(cnt), words;
    std::vector<int32_t> rfl(cnt);
    CK(cudaMemcpyAsync(res.data(), g.d_results, cnt * sizeof(SmallResult), cudaMemcpyDeviceToHost, g.st));
    CK(cudaMemcpyAsync(r64.data(), g.d_res64, cnt * sizeof(uint64_t), cudaMemcpyDeviceToHost, g.st));
    CK(cudaMemcpyAsync(rfl.data(), g.d_rflags, cnt * sizeof(int32_t), cudaMemcpyDeviceToHost, g.st));
    if (b->keep_words) {
        words.resize(g.total_words);
        CK(cudaMemcpyAsync(words.data(), g.d_words, g.total_words * sizeof(uint64_t), cudaMemcpyDeviceToHost, g.st));
    }
    CK(cudaStreamSynchronize(g.st));
    size_t woff = 0;
    for (size_t i = 0; i < cnt; ++i) {
        const Item& it = g.items[i];
        llg_result& r = b->out[it.idx];
        const size_t nw = (size_t)((it.p + 63) / 64);
        const size_t my_off = woff;
        woff += nw;
        r.max_err = std::max(r.max_err, res[i].max_err);
        r.seconds += (double)res[i].ns * 1e-9;
        if (res[i].status == LLG_ST_ROUNDOFF) {
            const uint32_t nn = next_fp64_length(it.p, n);
            r.n = n;
            r.escalations = it.escalations;
            if (!nn) {
                r.status = LLG_E_ROUNDOFF;
                continue;
            }
            Item again = it;
            again.n = nn;
            again.escalations++;
            retry.push_back(again);
            continue;
        }
        r.iters = res[i].iters_done;
        r.n = n;
        r.escalations = it.escalations;
        if (rfl[i] & 2) return fail(LLG_E_CUDA, "device residue rebuild did not settle (p=%llu)", (unsigned long long)it.p);
        if (b->keep_words) b->words[it.idx].assign(words.begin() + my_off, words.begin() + my_off + nw);
        r.res64 = r64[i];
        r.is_zero = (rfl[i] & 1) ? 1 : 0;
        r.status = LLG_OK;
    }
    return LLG_OK;
}

// Squarings between round-off checks (and residue snapshots) of the two-pass engines.
constexpr uint64_t kCheckChunk = 4096;

double bits_to_double(unsigned long long b) {
    double d;
    std::memcpy(&d, &b, sizeof d);
    return d;
}

// Shape of the two-pass FP64 engine per log2 N: row length (log2) and rows per row-pass block
// (-1 / 0: the built-in defaults); set by llg_set_large_split (the autotuner's choice). The two
// are packed in one word so a reader never sees half of an update.
std::atomic<int> g_large_shape[kLargeLogMax + 1];
struct SplitInit {
    SplitInit() {
        for (auto& x : g_large_shape) x.store(-1);
    }
} g_split_init;

int shape_log_c(int v) { return v < 0 ? -1 : v & 0xff; }
int shape_rows(int v) { return v < 0 ? 0 : v >> 8; }

cudaError_t init_large(LargeTest& T, uint64_t p, uint64_t n) {
    const int l = ilog2_exact(n);
    if (l < 0) return T.init(p, n);  // R0 2^k: fixed shape
    const int v = g_large_shape[l].load();
    return T.init(p, n, shape_log_c(v), shape_rows(v));
}

// The autotuners' choices (llgpu.autotune, llgpu.autotune_range) persist in a text file, one line
// per choice:
//   large_split <TAB> device name <TAB> log2 N <TAB> log2 row length <TAB> rows per block
//   length <TAB> device name <TAB> whole-test length of the rule <TAB> length to use instead
// read once per process from $LLG_TUNE_CACHE, else $HOME/.cache/llgpu/tune.txt. Lines for other
// devices or unsupported splits are ignored; llg_set_large_split overrides.
void load_tuning_once(int dev) {
    static std::once_flag once;
    std::call_once(once, [dev] {
        std::string path;
        if (const char* e = std::getenv("LLG_TUNE_CACHE")) path = e;
        else if (const char* h = std::getenv("HOME")) path = std::string(h) + "/.cache/llgpu/tune.txt";
        if (path.empty()) return;
        FILE* f = std::fopen(path.c_str(), "r");
        if (!f) return;
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
            std::fclose(f);
            return;
        }
        char line[512];
        while (std::fgets(line, sizeof line, f)) {
            char* fields[5] = {};
            int nf = 0;
            char* save = nullptr;
            for (char* tok = strtok_r(line, "\t\n", &save); tok && nf < 5; tok = strtok_r(nullptr, "\t\n", &save))
                fields[nf++] = tok;
            if (nf == 4 && std::strcmp(fields[0], "length") == 0 && std::strcmp(fields[1], prop.name) == 0) {
                const uint32_t nd = (uint32_t)std::strtoul(fields[2], nullptr, 10);
                const uint32_t nu = (uint32_t)std::strtoul(fields[3], nullptr, 10);
                const int i = length_index(nd);
                if (i >= 0 && is_small_length(nd) && length_index(nu) >= 0 && nu >= nd) g_length_choice[i].store(nu);
                continue;
            }
            if (nf != 5 || std::strcmp(fields[0], "large_split") != 0 || std::strcmp(fields[1], prop.name) != 0)
                continue;
            const int ln = std::atoi(fields[2]), lc = std::atoi(fields[3]), rows = std::atoi(fields[4]);
            if (large_split_supported(ln, lc, rows)) g_large_shape[ln].store(lc | (rows << 8));
        }
        std::fclose(f);
    });
}
cudaError_t init_large(NttLargeTest& T, uint64_t p, uint64_t n) { return T.init(p, ilog2_exact(n)); }

// The exact residue of a two-pass test's digits (on the device after its FINAL pass), rebuilt on
// the GPU; the words come back to the host only when asked for (into a vector or a caller buffer).
int device_residue(uint64_t p, uint32_t n, const int* d_digits, std::vector<uint64_t>* vec, uint64_t* host,
                   size_t host_cap, uint64_t* res64, int32_t* z, cudaStream_t st) {
    const size_t nw = (size_t)((p + 63) / 64);
    uint64_t* dw = nullptr;
    if (vec || host) CK(cudaMallocAsync(&dw, nw * sizeof(uint64_t), st));
    int rc = llg_residue_from_digits_device(p, n, d_digits, dw, res64, z, st);
    if (rc) rc = fail(rc, "residue rebuild on the device failed");
    if (!rc && dw) {
        uint64_t* dst = host;
        if (vec) {
            vec->assign(nw, 0);
            dst = vec->data();
        }
        if (cudaMemcpyAsync(dst, dw, nw * sizeof(uint64_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            rc = fail(LLG_E_CUDA, "copying the residue words back");
        if (host)
            for (size_t i = nw; i < host_cap; ++i) host[i] = 0;
    }
    if (dw) cudaFreeAsync(dw, st);
    if (rc) return rc;
    CK(cudaStreamSynchronize(st));
    return LLG_OK;
}

// The last two-pass test a single-exponent call ran, kept with its tables, buffers and captured
// graph for the next call on the same exponent, length, split and device: a repeated call (interim
// residues of one exponent, a driver's --verify pass) starts from the INIT pass instead of building
// tables, allocating ~30 bytes a digit and capturing graphs again. The reference keeps its FFTW
// plans per length the same way (lucaslehmer.cpp:229-242). One slot per engine; llg_release_cached
// frees it. Heap-held and never destroyed at exit (the CUDA context may be gone by then).
template <class TestT>
struct KeptTest {
    std::mutex mx;
    std::unique_ptr<TestT> t;
    uint64_t p = 0, n = 0;
    int shape = 0, dev = -1;
};
template <class TestT>
KeptTest<TestT>& kept() {
    static KeptTest<TestT>* k = new KeptTest<TestT>();
    return *k;
}
// the split init_large uses for (p, n) now (power-of-two FP64 lengths); -2 elsewhere
template <class TestT>
int kept_shape(uint64_t n) {
    if (!std::is_same<TestT, LargeTest>::value) return -2;
    const int l = ilog2_exact(n);
    return l < 0 ? -2 : g_large_shape[l].load();
}
template <class TestT>
std::unique_ptr<TestT> take_kept(uint64_t p, uint64_t n) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    KeptTest<TestT>& k = kept<TestT>();
    std::lock_guard<std::mutex> lk(k.mx);
    if (k.t && k.p == p && k.n == n && k.dev == dev && k.shape == kept_shape<TestT>(n)) return std::move(k.t);
    return nullptr;
}
template <class TestT>
void keep(std::unique_ptr<TestT> t, uint64_t p, uint64_t n) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    KeptTest<TestT>& k = kept<TestT>();
    std::unique_ptr<TestT> old;
    {
        std::lock_guard<std::mutex> lk(k.mx);
        old = std::move(k.t);
        k.t = std::move(t);
        k.p = p;
        k.n = n;
        k.dev = dev;
        k.shape = kept_shape<TestT>(n);
    }
}  // the test it replaces is freed here, outside the lock

// One exponent on a two-pass engine, in chunks of kCheckChunk squarings with a round-off check
// after each. FP64: after every chunk that stayed within the bound (and has more to go), the exact
// residue is rebuilt on the GPU into a device snapshot; a chunk above the bound is redone from the
// last snapshot at the next usable length (the words re-digitised there on the GPU), so an
// escalation repeats at most one chunk. r.seconds is the device time of every attempt.
template <class TestT>
int run_large_t(const Item& item, llg_result& r, std::vector<uint64_t>* words, cudaStream_t st) {
    constexpr bool kFp64 = std::is_same<TestT, LargeTest>::value;  // the NTT is exact: no checkpoints
    const uint64_t p = item.p;
    const size_t nw = (size_t)((p + 63) / 64);
    uint32_t n = item.n;
    uint32_t esc = item.escalations;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const double abort_err = g_abort_err.load();
    uint64_t* snap = nullptr;    // residue after snap_iters squarings (device words)
    uint64_t snap_iters = 0;     // 0: the snapshot is s_0 = 4 itself
    double total_ms = 0.0, worst = 0.0;
    auto cleanup = [&] {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (snap) cudaFreeAsync(snap, st);
    };
    auto bail = [&](int rc) {
        cleanup();
        return rc;
    };
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return bail(fail(LLG_E_CUDA, "creating events"));
    if (kFp64 && item.iters > kCheckChunk && cudaMallocAsync(&snap, nw * sizeof(uint64_t), st) != cudaSuccess)
        return bail(fail(LLG_E_NOMEM, "allocating the residue snapshot"));
    for (;;) {
        std::unique_ptr<TestT> held = take_kept<TestT>(p, n);
        cudaError_t ce = cudaSuccess;
        if (!held) {
            held.reset(new TestT());
            ce = init_large(*held, p, n);
        }
        TestT& T = *held;
        if (ce == cudaSuccess) ce = cudaEventRecord(e0, st);
        if (ce == cudaSuccess) {
            if (snap_iters == 0) {
                ce = T.start_seed(st);
            } else {
                ce = digits_from_words(p, n, snap, T.digits, st);
                if (ce == cudaSuccess) ce = T.start_device(st);
            }
        }
        if (ce != cudaSuccess) return bail(fail(ce == cudaErrorMemoryAllocation ? LLG_E_NOMEM : LLG_E_CUDA, "CUDA: %s", cudaGetErrorString(ce)));
        uint64_t done = snap_iters + 1;
        bool abort = false;
        double err = 0.0;
        while (done < item.iters && !abort) {
            const uint64_t k = std::min(item.iters - done, kCheckChunk);
            LargeCtl h;
            ce = T.step(k, st);
            if (ce == cudaSuccess) ce = T.read_ctl(h, st);
            if (ce != cudaSuccess) return bail(fail(LLG_E_CUDA, "CUDA: %s", cudaGetErrorString(ce)));
            if (h.timeout) return bail(fail(LLG_E_TIMEOUT, "carry wait timed out (p=%llu)", (unsigned long long)p));
            done += k;
            err = bits_to_double(h.err_max);
            if (err > abort_err) {
                abort = true;
            } else if (kFp64 && snap && done < item.iters) {
                // checkpoint: the exact residue of this clean state, kept on the device
                ce = T.final_pass(st);
                if (ce != cudaSuccess) return bail(fail(LLG_E_CUDA, "CUDA: %s", cudaGetErrorString(ce)));
                int32_t z = 0;
                uint64_t r64 = 0;
                const int rc = llg_residue_from_digits_device(p, n, T.digits, snap, &r64, &z, st);
                if (rc) return bail(fail(rc, "residue snapshot on the device failed"));
                snap_iters = done;
            }
        }
        if (!abort) {
            LargeCtl h;
            ce = T.final_pass(st);
            if (ce == cudaSuccess) ce = cudaEventRecord(e1, st);
            if (ce == cudaSuccess) ce = T.read_ctl(h, st);
            if (ce != cudaSuccess) return bail(fail(LLG_E_CUDA, "CUDA: %s", cudaGetErrorString(ce)));
            if (h.timeout) return bail(fail(LLG_E_TIMEOUT, "carry wait timed out (p=%llu)", (unsigned long long)p));
            err = bits_to_double(h.err_max);
            if (err > abort_err) abort = true;
        } else if (cudaEventRecord(e1, st) != cudaSuccess) {
            return bail(fail(LLG_E_CUDA, "recording an event"));
        }
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
            return bail(fail(LLG_E_CUDA, "timing the attempt"));
        total_ms += ms;
        worst = std::max(worst, err);
        const uint32_t n_ran = n;
        if (abort) {  // FP64 only: the NTT's round-off is identically zero
            const uint32_t nn = next_fp64_length(p, n);
            if (!nn) {
                r.status = LLG_E_ROUNDOFF;
                r.n = n;
                r.escalations = esc;
                r.max_err = worst;
                break;
            }
            n = nn;
            ++esc;
            continue;
        }
        int32_t z = 0;
        const int rc = device_residue(p, n, T.digits, words, nullptr, 0, &r.res64, &z, st);
        if (rc) return bail(rc);
        keep(std::move(held), p, n_ran);  // idle: device_residue waited for the stream
        r.iters = item.iters;
        r.is_zero = z;
        r.n = n;
        r.escalations = esc;
        r.seconds = total_ms * 1e-3;
        r.max_err = err;  // the round-off of the attempt that produced the result
        r.status = LLG_OK;
        break;
    }
    cleanup();
    return LLG_OK;
}

int run_large(int engine, const Item& item, llg_result& r, std::vector<uint64_t>* words, cudaStream_t st) {
    return engine == LLG_ENGINE_NTT ? run_large_t<NttLargeTest>(item, r, words, st)
                                    : run_large_t<LargeTest>(item, r, words, st);
}

// Creates a batch: trivial exponents resolved on the host, the rest grouped by length.
// strict: a single-exponent call fails on an unsupported exponent; a batch marks it and goes on
// (the reference's batch returns such exponents with seconds < 0, cuda/ll_ntt.cu:259-267).
int make_batch(const uint64_t* ps, size_t count, uint64_t max_iters, int engine, uint32_t n_force,
               bool strict, int flags, llg_batch** outb, const uint64_t* iters_each = nullptr) {
    if (engine != LLG_ENGINE_FP64 && engine != LLG_ENGINE_NTT) return fail(LLG_E_ARG, "unknown engine %d", engine);
    const bool ntt = engine == LLG_ENGINE_NTT;
    int dev;
    int rc = device_ready(&dev);
    if (rc) return rc;
    llg_batch* b = new llg_batch();
    b->dev = dev;
    b->engine = engine;
    b->count = count;
    b->ps.assign(ps, ps + count);
    b->out.resize(count);
    b->keep_words = (flags & LLG_BATCH_KEEP_WORDS) != 0;
    if (b->keep_words) b->words.resize(count);
    std::map<uint32_t, std::vector<Item>> groups;
    for (size_t i = 0; i < count; ++i) {
        const uint64_t p = ps[i];
        set_trivial(&b->out[i], p);
        if (p < 3 || p % 2 == 0) continue;  // decided without iterating (lucaslehmer.cpp:31-33)
        const uint64_t full = p - 2;
        const uint64_t mi = iters_each ? iters_each[i] : max_iters;
        const uint64_t iters = (mi && mi < full) ? mi : full;
        b->out[i].iters = iters;
        Item it{i, p, iters, 0, 0};
        if (p >= kWordMaxP) {
            uint32_t n = n_force;
            if (n_force && !(ntt ? ntt_length_usable(p, n_force) : fp64_length_usable(p, n_force))) {
                destroy_batch(b);
                return fail(LLG_E_UNSUPPORTED, "length %u not usable for p=%llu", n_force, (unsigned long long)p);
            }
            if (!n) n = ntt ? ntt_len(p) : fp64_length(p, g_max_bpw);
            if (!n) {
                b->out[i].status = LLG_E_UNSUPPORTED;
                if (strict) {
                    destroy_batch(b);
                    return fail(LLG_E_UNSUPPORTED, "p=%llu above the engine's range", (unsigned long long)p);
                }
                continue;
            }
            it.n = n;
        }
        if (it.n && !is_small_length(it.n))
            b->large.push_back(it);
        else
            groups[it.n].push_back(it);
    }
    for (auto& kv : groups) {
        Group g;
        g.n = kv.first;
        g.items = std::move(kv.second);
        b->groups.push_back(std::move(g));
    }
    // largest lengths first (they run longest)
    std::sort(b->groups.begin(), b->groups.end(), [](const Group& x, const Group& y) { return x.n > y.n; });
    for (Group& g : b->groups) {
        if ((rc = setup_group(g, b->keep_words))) {
            destroy_batch(b);
            return rc;
        }
    }
    cudaError_t e = cudaEventCreate(&b->fork);
    if (e == cudaSuccess) e = cudaEventCreate(&b->joined);
    if (e == cudaSuccess && (flags & LLG_BATCH_ERRLOG) && b->groups.size() == 1 &&
        b->groups[0].items.size() == 1 && b->groups[0].n) {
        b->errlog_len = b->groups[0].items[0].iters;
        e = cudaMalloc(&b->d_errlog, b->errlog_len * sizeof(float));
        if (e == cudaSuccess) e = cudaMemset(b->d_errlog, 0, b->errlog_len * sizeof(float));
    }
    if (e != cudaSuccess) {
        destroy_batch(b);
        return fail(LLG_E_CUDA, "CUDA: %s", cudaGetErrorString(e));
    }
    *outb = b;
    return LLG_OK;
}

int launch_batch(llg_batch* b, cudaStream_t caller) {
    for (const Group& g : b->groups)
        for (const Item& it : g.items) {
            b->out[it.idx].seconds = 0.0;
            b->out[it.idx].max_err = 0.0;
        }
    CK(cudaEventRecord(b->fork, caller));
    for (Group& g : b->groups) {
        int rc = launch_group(b, g, caller);
        if (rc) return rc;
    }
    CK(cudaEventRecord(b->joined, caller));
    b->launched = true;
    return LLG_OK;
}

// Collects every group; round-off aborts are rerun (synchronously) at longer lengths until done.
int collect_batch(llg_batch* b) {
    if (b->collected) return LLG_OK;
    std::vector<Item> retry;
    for (Group& g : b->groups) {
        int rc = collect_group(b, g, retry);
        if (rc) return rc;
    }
    std::vector<Item> large = b->large;
    for (int round = 0; !retry.empty() && round < 16; ++round) {
        std::map<uint32_t, std::vector<Item>> byn;
        for (Item& it : retry) {
            if (it.n && !is_small_length(it.n))
                large.push_back(it);
            else
                byn[it.n].push_back(it);
        }
        retry.clear();
        for (auto& kv : byn) {
            Group g;
            g.n = kv.first;
            g.items = std::move(kv.second);
            int rc = setup_group(g, b->keep_words);
            if (!rc) {
                CK(cudaEventRecord(b->fork, g.st));
                rc = launch_group(b, g, g.st);
            }
            if (!rc) rc = collect_group(b, g, retry);
            release_group(g);
            if (rc) return rc;
        }
    }
    if (!large.empty()) {
        cudaStream_t st = b->groups.empty() ? nullptr : b->groups[0].st;
        cudaStream_t own = nullptr;
        if (!st) {
            CK(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
            st = own;
        }
        for (const Item& it : large) {
            const int rc = run_large(b->engine, it, b->out[it.idx], b->keep_words ? &b->words[it.idx] : nullptr, st);
            if (rc) {
                if (own) cudaStreamDestroy(own);
                return rc;
            }
        }
        if (own) cudaStreamDestroy(own);
    }
    b->collected = true;
    return LLG_OK;
}

cudaStream_t default_stream_for_thread() {
    static thread_local cudaStream_t st = nullptr;
    static thread_local int dev = -1;
    int d = -1;
    cudaGetDevice(&d);
    if (!st || dev != d) {
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        dev = d;
    }
    return st;
}

int run_sync(llg_batch* b) {
    cudaStream_t st = default_stream_for_thread();
    int rc = launch_batch(b, st);
    if (rc) return rc;
    return collect_batch(b);
}

// ---- single-exponent calls from many host threads share batches ------------------------------
// The reference's driver tests one exponent per call from a thread pool (PerfNumMultiCLL.py:34-42,
// 174-193). llg_run calls whose length is a whole-test length join a per-device pool instead of
// each making its own one-block launch: the first caller of a round leads it -- it waits
// kGatherWindow for the calls arriving meanwhile, takes every pending request, runs them as one
// batch (one launch per transform length), hands each caller its result and wakes it; a request
// that arrived during the round leads the next one. The window is short while callers come one at
// a time (the previous round held one request) and longer once several call at once.
constexpr auto kGatherWindow = std::chrono::microseconds(150);
constexpr auto kGatherWindowAlone = std::chrono::microseconds(10);

struct Request {
    uint64_t p = 0, iters = 0;
    int engine = 0;
    bool want_words = false;
    llg_result res{};
    std::vector<uint64_t> words;
    int rc = LLG_OK;
    std::string err;
    bool done = false, lead = false;
};

struct CallPool {
    std::mutex mx;
    std::condition_variable cv;
    std::vector<Request*> pending;
    bool leading = false;
    size_t last_round = 1;  // requests in the previous round
};

std::mutex g_pools_mx;
std::map<int, std::unique_ptr<CallPool>> g_pools;  // per device ordinal

CallPool& call_pool(int dev) {
    std::lock_guard<std::mutex> lk(g_pools_mx);
    std::unique_ptr<CallPool>& p = g_pools[dev];
    if (!p) p.reset(new CallPool());
    return *p;
}

int run_sync(llg_batch* b);
void destroy_batch(llg_batch* b);

// One round: every request of `reqs`, one batch per engine.
void run_round(std::vector<Request*>& reqs) {
    for (int engine : {LLG_ENGINE_FP64, LLG_ENGINE_NTT}) {
        std::vector<Request*> mine;
        for (Request* r : reqs)
            if (r->engine == engine) mine.push_back(r);
        if (mine.empty()) continue;
        std::vector<uint64_t> ps, its;
        bool words = false;
        for (Request* r : mine) {
            ps.push_back(r->p);
            its.push_back(r->iters);
            words = words || r->want_words;
        }
        llg_batch* b = nullptr;
        int rc = make_batch(ps.data(), ps.size(), 0, engine, 0, false, words ? LLG_BATCH_KEEP_WORDS : 0, &b, its.data());
        if (!rc) rc = run_sync(b);
        std::vector<llg_result> out(ps.size());
        std::vector<uint64_t> wbuf;
        if (!rc) {
            size_t total = 0;
            for (uint64_t p : ps) total += (size_t)((p + 63) / 64);
            if (words) wbuf.resize(total);
            rc = llg_batch_results(b, out.data(), words ? wbuf.data() : nullptr, wbuf.size());
        }
        if (b) destroy_batch(b);
        size_t off = 0;
        for (size_t i = 0; i < mine.size(); ++i) {
            Request* r = mine[i];
            const size_t nw = (size_t)((r->p + 63) / 64);
            r->rc = rc;
            if (rc) r->err = t_last_error;
            else r->res = out[i];
            if (!rc && r->want_words) r->words.assign(wbuf.begin() + off, wbuf.begin() + off + nw);
            off += nw;
        }
    }
}

// Runs `r` through the device's pool; returns when its result is in.
void run_pooled(int dev, Request& r) {
    CallPool& P = call_pool(dev);
    std::unique_lock<std::mutex> lk(P.mx);
    P.pending.push_back(&r);
    if (!P.leading) {
        P.leading = true;
        r.lead = true;
    }
    P.cv.wait(lk, [&] { return r.done || r.lead; });
    if (r.done) return;
    // lead this round
    const auto window = P.last_round > 1 ? kGatherWindow : kGatherWindowAlone;
    lk.unlock();
    std::this_thread::sleep_for(window);
    lk.lock();
    std::vector<Request*> round;
    round.swap(P.pending);
    P.last_round = round.size();
    lk.unlock();
    run_round(round);
    lk.lock();
    for (Request* q : round) q->done = true;
    if (!P.pending.empty()) P.pending.front()->lead = true;
    else P.leading = false;
    P.cv.notify_all();
}

}  // namespace

namespace llg {
int set_error(int code, const char* msg) { return fail(code, "%s", msg); }
std::atomic<uint64_t> g_h2d_bytes{0};
void count_h2d(size_t bytes) { g_h2d_bytes.fetch_add((uint64_t)bytes, std::memory_order_relaxed); }
}  // namespace llg

extern "C" uint64_t llg_h2d_bytes(void) { return llg::g_h2d_bytes.load(); }

extern "C" void llg_release_cached(void) {
    keep<LargeTest>(nullptr, 0, 0);
    keep<NttLargeTest>(nullptr, 0, 0);
}

extern "C" {

const char* llg_status_string(int s) {
    switch (s) {
        case LLG_OK: return "ok";
        case LLG_E_CUDA: return "CUDA error";
        case LLG_E_NODEV: return "no CUDA device";
        case LLG_E_ARG: return "invalid argument";
        case LLG_E_UNSUPPORTED: return "unsupported exponent or length";
        case LLG_E_ROUNDOFF: return "round-off above threshold at every length";
        case LLG_E_TIMEOUT: return "device wait timed out";
        case LLG_E_NOMEM: return "device out of memory";
        default: return "unknown status";
    }
}

const char* llg_last_error(void) { return t_last_error.c_str(); }

int llg_device_info(char* name, size_t cap, int* sms, uint64_t* mem) {
    int dev;
    int rc = device_ready(&dev);
    if (rc) return rc;
    cudaDeviceProp pr;
    CK(cudaGetDeviceProperties(&pr, dev));
    if (name && cap) {
        std::strncpy(name, pr.name, cap - 1);
        name[cap - 1] = 0;
    }
    if (sms) *sms = pr.multiProcessorCount;
    if (mem) *mem = (uint64_t)pr.totalGlobalMem;
    return LLG_OK;
}

uint32_t llg_fft_length(uint64_t p, double max_bpw) {
    if (max_bpw <= 0) max_bpw = g_max_bpw;
    if (p < kWordMaxP) return 0;
    return fp64_length(p, max_bpw);
}

int llg_set_large_split(int log_n, int log_c, int rows) {
    if (!large_length_supported(log_n)) return fail(LLG_E_ARG, "log2 N = %d is not a two-pass length", log_n);
    if (log_c < 0) {
        g_large_shape[log_n].store(-1);
        return LLG_OK;
    }
    if (!large_split_supported(log_n, log_c, rows))
        return fail(LLG_E_UNSUPPORTED, "no kernels for rows of 2^%d, %d per block, at N = 2^%d", log_c, rows, log_n);
    g_large_shape[log_n].store(log_c | ((rows ? rows : large_rows_per_block(log_c)) << 8));
    return LLG_OK;
}

int llg_get_large_split(int log_n, int* rows) {
    if (!large_length_supported(log_n)) return -1;
    const int v = g_large_shape[log_n].load();
    const int lc = v >= 0 ? shape_log_c(v) : large_default_log_c(log_n);
    if (rows) *rows = v >= 0 ? shape_rows(v) : large_rows_per_block(lc);
    return lc;
}

int llg_set_length_choice(uint32_t n_rule, uint32_t n_use) {
    const int i = length_index(n_rule);
    if (i < 0 || !is_small_length(n_rule)) return fail(LLG_E_ARG, "%u is not a whole-test FP64 length", n_rule);
    if (n_use && (length_index(n_use) < 0 || n_use < n_rule))
        return fail(LLG_E_ARG, "%u is not an FP64 length at least %u", n_use, n_rule);
    g_length_choice[i].store(n_use == n_rule ? 0u : n_use);
    return LLG_OK;
}

uint32_t llg_get_length_choice(uint32_t n_rule) {
    const int i = length_index(n_rule);
    const uint32_t c = i >= 0 ? g_length_choice[i].load() : 0u;
    return c ? c : n_rule;
}

int llg_set_roundoff_limit(double limit) {
    if (!(limit > 0.0 && limit < 0.5)) return fail(LLG_E_ARG, "round-off limit %g outside (0, 0.5)", limit);
    g_abort_err.store(limit);
    return LLG_OK;
}

double llg_get_roundoff_limit(void) { return g_abort_err.load(); }

int llg_set_max_bpw(double b) {
    if (!(b >= 2.0 && b <= (double)kMaxDigitBits)) return fail(LLG_E_ARG, "bits per word %g out of range [2, 28]", b);
    g_max_bpw = b;
    return LLG_OK;
}

double llg_get_max_bpw(void) { return g_max_bpw; }

uint32_t llg_ntt_length(uint64_t p) { return ntt_len(p); }

uint64_t llg_max_exponent(int engine) {
    if (engine == LLG_ENGINE_FP64) return (uint64_t)std::floor(g_max_bpw * (double)(1u << kLargeLogMax));
    if (engine == LLG_ENGINE_NTT) return (uint64_t)((63 - kLargeLogMax) / 2) << kLargeLogMax;
    return 0;
}

int llg_run(uint64_t p, uint64_t max_iters, int engine, uint32_t n, llg_result* out,
            uint64_t* words, size_t nwords) {
    if (!out) return fail(LLG_E_ARG, "null result pointer");
    const size_t nw = (size_t)((p + 63) / 64);
    if (words && nwords < nw) return fail(LLG_E_ARG, "words buffer too small (%zu < %zu)", nwords, nw);
    if (n == 0 && (engine == LLG_ENGINE_FP64 || engine == LLG_ENGINE_NTT)) {
        // whole-test lengths (and the word path): share a batch with concurrent callers
        const uint32_t len = p < kWordMaxP ? 0 : (engine == LLG_ENGINE_NTT ? ntt_len(p) : fp64_length(p, g_max_bpw));
        if (p < kWordMaxP || (len && is_small_length(len))) {
            int dev;
            int rc = device_ready(&dev);
            if (rc) return rc;
            Request r;
            r.p = p;
            r.iters = max_iters;
            r.engine = engine;
            r.want_words = words != nullptr;
            run_pooled(dev, r);
            if (r.rc) return fail(r.rc, "%s", r.err.c_str());
            *out = r.res;
            if (words) {
                std::memset(words, 0, nwords * sizeof(uint64_t));
                std::memcpy(words, r.words.data(), std::min(nw, r.words.size()) * sizeof(uint64_t));
            }
            if (out->status) return fail(out->status, "p=%llu: %s", (unsigned long long)p, llg_status_string(out->status));
            return LLG_OK;
        }
    }
    llg_batch* b = nullptr;
    int rc = make_batch(&p, 1, max_iters, engine, n, true, words ? LLG_BATCH_KEEP_WORDS : 0, &b);
    if (rc) return rc;
    rc = run_sync(b);
    if (!rc) rc = llg_batch_results(b, out, words, nwords);
    destroy_batch(b);
    if (rc) return rc;
    return out->status;
}

int llg_run_batch(const uint64_t* ps, size_t count, uint64_t max_iters, int engine,
                  llg_result* out, uint64_t* words_out, size_t words_cap) {
    if (!out || (!ps && count)) return fail(LLG_E_ARG, "null pointer");
    if (count == 0) return LLG_OK;
    llg_batch* b = nullptr;
    int rc = make_batch(ps, count, max_iters, engine, 0, false, words_out ? LLG_BATCH_KEEP_WORDS : 0, &b);
    if (rc) return rc;
    rc = run_sync(b);
    if (!rc) rc = llg_batch_results(b, out, words_out, words_cap);
    destroy_batch(b);
    return rc;
}

int llg_batch_create(const uint64_t* ps, size_t count, uint64_t max_iters, int engine, int flags,
                     llg_batch** out) {
    if (!out || !ps || count == 0) return fail(LLG_E_ARG, "null pointer or empty batch");
    *out = nullptr;
    return make_batch(ps, count, max_iters, engine, 0, false, flags, out);
}

int llg_batch_launch(llg_batch* b, void* stream) {
    if (!b) return fail(LLG_E_ARG, "null batch");
    cudaStream_t st = stream ? (cudaStream_t)stream : default_stream_for_thread();
    b->collected = false;
    return launch_batch(b, st);
}

int llg_batch_results(llg_batch* b, llg_result* out, uint64_t* words, size_t words_cap) {
    if (!b || !out) return fail(LLG_E_ARG, "null pointer");
    if (!b->launched) return fail(LLG_E_ARG, "batch not launched");
    int rc = collect_batch(b);
    if (rc) return rc;
    std::memcpy(out, b->out.data(), b->count * sizeof(llg_result));
    if (words) {
        size_t total = 0;
        for (size_t i = 0; i < b->count; ++i) total += (size_t)((b->ps[i] + 63) / 64);
        if (words_cap < total) return fail(LLG_E_ARG, "words buffer too small (%zu < %zu)", words_cap, total);
        if (!b->keep_words) return fail(LLG_E_ARG, "batch created without LLG_BATCH_KEEP_WORDS");
        std::memset(words, 0, words_cap * sizeof(uint64_t));
        size_t off = 0;
        for (size_t i = 0; i < b->count; ++i) {
            const size_t nw = (size_t)((b->ps[i] + 63) / 64);
            const std::vector<uint64_t>& w = b->words[i];
            std::memcpy(words + off, w.data(), std::min(nw, w.size()) * sizeof(uint64_t));
            off += nw;
        }
    }
    return LLG_OK;
}

int llg_batch_errlog(llg_batch* b, float* log, size_t cap, size_t* len) {
    if (!b || !log) return fail(LLG_E_ARG, "null pointer");
    if (!b->d_errlog) return fail(LLG_E_ARG, "batch created without LLG_BATCH_ERRLOG (single exponent)");
    const size_t n = std::min(cap, (size_t)b->errlog_len);
    CK(cudaMemcpy(log, b->d_errlog, n * sizeof(float), cudaMemcpyDeviceToHost));
    if (len) *len = n;
    return LLG_OK;
}

int llg_batch_device_ms(llg_batch* b, float* ms) {
    if (!b || !ms) return fail(LLG_E_ARG, "null pointer");
    if (!b->launched) return fail(LLG_E_ARG, "batch not launched");
    CK(cudaEventSynchronize(b->joined));
    CK(cudaEventElapsedTime(ms, b->fork, b->joined));
    return LLG_OK;
}

void llg_batch_destroy(llg_batch* b) { destroy_batch(b); }

}  // extern "C"

struct llg_test {
    std::unique_ptr<llg::LargeTest> f;     // FP64 engine
    std::unique_ptr<llg::NttLargeTest> n;  // NTT engine
    int dev = -1;
    uint64_t p() const { return f ? f->p : n->p; }
    uint64_t len() const { return f ? f->N : n->N; }
    uint64_t done() const { return f ? f->done : n->done; }
};

extern "C" {

int llg_test_create(uint64_t p, uint32_t n, int engine, llg_test** out) {
    if (!out) return fail(LLG_E_ARG, "null pointer");
    *out = nullptr;
    if (engine != LLG_ENGINE_FP64 && engine != LLG_ENGINE_NTT) return fail(LLG_E_ARG, "unknown engine %d", engine);
    int dev;
    int rc = device_ready(&dev);
    if (rc) return rc;
    if (p < 3 || p % 2 == 0) return fail(LLG_E_ARG, "p must be odd and >= 3");
    const bool ntt = engine == LLG_ENGINE_NTT;
    if (n == 0) n = ntt ? ntt_len(p) : fp64_length(p, g_max_bpw);
    const int l = ilog2_exact(n);
    const bool ok = ntt ? (l > kSmallLogMax && ntt_large_length_supported(l) && ntt_length_usable(p, n))
                        : (large_fp64_length(n) && fp64_length_usable(p, n));
    if (!ok)
        return fail(LLG_E_UNSUPPORTED, "length %u not usable by the two-pass %s engine for p=%llu", n,
                    ntt ? "NTT" : "FP64", (unsigned long long)p);
    llg_test* t = new llg_test();
    t->dev = dev;
    cudaError_t e;
    if (ntt) {
        t->n.reset(new llg::NttLargeTest());
        e = t->n->init(p, l);
    } else {
        t->f.reset(new llg::LargeTest());
        e = init_large(*t->f, p, n);
    }
    if (e != cudaSuccess) {
        delete t;
        return fail(e == cudaErrorMemoryAllocation ? LLG_E_NOMEM : LLG_E_CUDA, "CUDA: %s", cudaGetErrorString(e));
    }
    *out = t;
    return LLG_OK;
}

int llg_test_start(llg_test* t, void* stream) {
    if (!t) return fail(LLG_E_ARG, "null test");
    cudaStream_t st = stream ? (cudaStream_t)stream : default_stream_for_thread();
    if (t->f) CK(t->f->start_seed(st));
    else CK(t->n->start_seed(st));
    return LLG_OK;
}

int llg_test_iterate(llg_test* t, uint64_t iters, void* stream) {
    if (!t) return fail(LLG_E_ARG, "null test");
    cudaStream_t st = stream ? (cudaStream_t)stream : default_stream_for_thread();
    if (t->f) CK(t->f->step(iters, st));
    else CK(t->n->step(iters, st));
    return LLG_OK;
}

int llg_test_read(llg_test* t, void* stream, llg_result* out, uint64_t* words, size_t nwords) {
    if (!t || !out) return fail(LLG_E_ARG, "null pointer");
    const uint64_t p = t->p();
    const size_t nw = (size_t)((p + 63) / 64);
    if (words && nwords < nw) return fail(LLG_E_ARG, "words buffer too small");
    cudaStream_t st = stream ? (cudaStream_t)stream : default_stream_for_thread();
    LargeCtl h;
    if (t->f) {
        CK(t->f->final_pass(st));
        CK(t->f->read_ctl(h, st));
    } else {
        CK(t->n->final_pass(st));
        CK(t->n->read_ctl(h, st));
    }
    std::memset(out, 0, sizeof *out);
    out->p = p;
    out->iters = t->done();
    out->n = (uint32_t)t->len();
    out->max_err = bits_to_double(h.err_max);
    if (h.timeout) return fail(LLG_E_TIMEOUT, "carry wait timed out");
    int32_t z = 0;
    const int* dd = t->f ? t->f->digits : t->n->digits;
    const int rc = device_residue(p, out->n, dd, nullptr, words, words ? nwords : 0, &out->res64, &z, st);
    if (rc) return rc;
    out->is_zero = z;
    out->status = out->max_err > g_abort_err.load() ? LLG_E_ROUNDOFF : LLG_OK;
    return LLG_OK;
}

int llg_test_time_passes(llg_test* t, uint64_t iters, void* stream, double* row_us, double* col_us) {
    if (!t || !row_us || !col_us) return fail(LLG_E_ARG, "null pointer");
    cudaStream_t st = stream ? (cudaStream_t)stream : default_stream_for_thread();
    if (t->f) CK(t->f->time_passes(iters, st, *row_us, *col_us));
    else CK(t->n->time_passes(iters, st, *row_us, *col_us));
    return LLG_OK;
}

int llg_test_load(llg_test* t, const uint64_t* words, size_t nwords, uint64_t iters_done, void* stream) {
    if (!t || !words) return fail(LLG_E_ARG, "null pointer");
    const uint64_t p = t->p();
    const size_t nw = (size_t)((p + 63) / 64);
    if (nwords < nw) return fail(LLG_E_ARG, "words buffer too small (%zu < %zu)", nwords, nw);
    if (p % 64 && (words[nw - 1] >> (p % 64)) != 0) return fail(LLG_E_ARG, "residue has bits at or above p");
    cudaStream_t st = stream ? (cudaStream_t)stream : default_stream_for_thread();
    uint64_t* dw = nullptr;
    CK(cudaMallocAsync(&dw, nw * sizeof(uint64_t), st));
    cudaError_t e = cudaMemcpyAsync(dw, words, nw * sizeof(uint64_t), cudaMemcpyHostToDevice, st);
    count_h2d(nw * sizeof(uint64_t));
    int* digits = t->f ? t->f->digits : t->n->digits;
    if (e == cudaSuccess) e = digits_from_words(p, t->len(), dw, digits, st);
    if (e == cudaSuccess) e = t->f ? t->f->start_device(st) : t->n->start_device(st);
    cudaFreeAsync(dw, st);
    if (e != cudaSuccess) return fail(LLG_E_CUDA, "CUDA: %s", cudaGetErrorString(e));
    if (t->f) t->f->done = iters_done + 1;
    else t->n->done = iters_done + 1;
    return LLG_OK;
}

int llg_test_diag_withhold_wrap(llg_test* t, uint64_t spin_limit, void* stream) {
    if (!t) return fail(LLG_E_ARG, "null test");
    if (!t->f) return fail(LLG_E_ARG, "the withheld-wrap diagnostic is for the FP64 engine");
    cudaStream_t st = stream ? (cudaStream_t)stream : default_stream_for_thread();
    bool timed_out = false;
    CK(t->f->diag_withhold_wrap(spin_limit, st, timed_out));
    if (timed_out) return fail(LLG_E_TIMEOUT, "carry wait timed out (wrap-around job withheld)");
    return LLG_OK;
}

int llg_test_errlog(llg_test* t, float* log, size_t cap, size_t* len) {
    if (!t || !log) return fail(LLG_E_ARG, "null pointer");
    if (!t->f) return fail(LLG_E_ARG, "the NTT engine has no round-off log (it is exact)");
    const size_t have = (size_t)std::min<uint64_t>(t->f->done, (uint64_t)t->f->errlog_len);
    const size_t n = std::min(cap, have);
    // the squarings may still run on any stream: wait for the device before reading the log
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(log, t->f->errlog, n * sizeof(float), cudaMemcpyDeviceToHost));
    if (len) *len = n;
    return LLG_OK;
}

void llg_test_destroy(llg_test* t) { delete t; }

}  // extern "C"
