// Host side of the two-pass engine: per-test device state, tables, the launch sequence of a
// squaring (row pass, column pass), CUDA-graph capture of chunks of squarings, read-back.
//
// Launch sequence for k squarings from given digits:  row(INIT), col, [row(ITER), col] x (k-1),
// row(FINAL). Every row pass after the first finishes the previous squaring (inverse row FFT,
// carry) and starts the next (forward row FFT); every column pass is one pointwise square.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>

#include "../../include/llgpu.h"
#include "llg_device.cuh"
#include "llg_host.h"
#include "llg_internal.h"

namespace llg {

namespace {

// column slot of row-FFT frequency k
int host_pos_of_freq(int log_l, int LE, int k) {
    // digit reversal of the row FFT's output positions (radix 2^LE passes, the last one RLAST):
    // host copy of pos_of_freq for SmallGeom<log_l, LE>
    const int E = 1 << LE;
    const int L = 1 << log_l, P = (log_l + LE - 1) / LE;
    const int RLAST = (log_l % LE == 0) ? E : (1 << (log_l % LE));
    const int klast = k / (L / RLAST);
    int low = k % (L / RLAST), rest = 0;
    for (int q = 0; q < P - 1; ++q) {
        rest = (rest << LE) | (low & (E - 1));
        low >>= LE;
    }
    return rest * RLAST + klast;
}

std::vector<double2> omega_table(uint64_t period, uint64_t count, uint64_t step) {
    // e^{-2 pi i x step / period}, x < count, rounded once from long double
    std::vector<double2> t(count);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (uint64_t x = 0; x < count; ++x) {
        const uint64_t e = (x * step) % period;
        const long double ang = two_pi * (long double)e / (long double)period;
        t[x] = make_double2((double)cosl(ang), -(double)sinl(ang));
    }
    return t;
}

template <class T>
cudaError_t upload(T** d, const std::vector<T>& h);

}  // namespace

double2 padded_quarter_slot(uint64_t L, uint64_t i) {
    if (i % 9 == 8) return make_double2(0.0, 0.0);
    const uint64_t r = 8 * (i / 9) + (i % 9);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    const long double ang = two_pi * (long double)r / (long double)L;
    return make_double2((double)cosl(ang), -(double)sinl(ang));
}

std::vector<double2> spread_quarter_table(uint64_t L) {
    const uint32_t qm = (uint32_t)(L / 4);
    std::vector<double2> t(qpad_s_len(qm), make_double2(0.0, 0.0));
    // entry r holds the value slot qpad(r) holds in the padded layout (the same long-double sum)
    for (uint32_t r = 0; r < qm; ++r) t[qpad_s(r)] = padded_quarter_slot(L, qpad(r));
    return t;
}

std::vector<double2> padded_quarter_table(uint64_t L) {
    const uint64_t n = qpad_len((uint32_t)(L / 4));
    std::vector<double2> t(n);
    for (uint64_t i = 0; i < n; ++i) t[i] = padded_quarter_slot(L, i);
    return t;
}

// Every e^{-2 pi i r / L}, r < L, at slot qpad(r) (the row FFT's table: no quadrant fold).
std::vector<double2> padded_full_table(uint64_t L) {
    const uint64_t n = qpad_len((uint32_t)L);
    std::vector<double2> t(n);
    for (uint64_t i = 0; i < n; ++i) t[i] = padded_quarter_slot(L, i);
    return t;
}

namespace {

template <class T>
cudaError_t upload(T** d, const std::vector<T>& h) {
    cudaError_t e = cudaMalloc(d, h.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    count_h2d(h.size() * sizeof(T));
    return cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
}

}  // namespace

bool large_length_supported(int log_n) { return log_n >= 14 && log_n <= 23; }

// The non-power-of-two two-pass lengths N = R0 2^k (R0 = 3, 5; k = 18 .. 21): columns of
// R = R0 2^9 complex values (large_col_mixed), rows of 2^(k - 10). Below k = 18 the C / 2 + 1
// column-pair blocks (65 or fewer) leave most of the GPU idle and the next power of two is faster.
bool large_mixed_length_supported(uint64_t n, int* r0, int* log_c) {
    for (int r = 3; r <= 5; r += 2) {
        if (n % (uint64_t)r) continue;
        const uint64_t m = n / (uint64_t)r;
        if (m & (m - 1)) continue;
        int k = 0;
        while ((1ull << k) < m) ++k;
        if (k < 18 || k > 21) return false;
        if (r0) *r0 = r;
        if (log_c) *log_c = k - 10;
        return true;
    }
    return false;
}

// Row length (2^log_c complex values) of the two-pass FP64 engine at N = 2^log_n by default.
int large_default_log_c(int log_n) {
    return (log_n <= 15) ? log_n - 8 : (log_n <= 17) ? 8 : (log_n <= 19) ? 9 : 10;
}

// Shapes of M = N/2 = 2^log_r rows of 2^log_c values (row blocks of `rows` rows) that the
// kernels implement: rows of 2^6 .. 2^11, columns of 2^7 .. 2^12; rows == 0: the default.
bool large_split_supported(int log_n, int log_c, int rows) {
    const int log_r = log_n - 1 - log_c;
    if (rows == 0) rows = large_rows_per_block(log_c);
    return large_length_supported(log_n) && log_r >= 7 && log_r <= 12 && large_rows_supported(log_c, rows);
}

LargeTest::~LargeTest() {
    if (exec) cudaGraphExecDestroy(exec);
    void* ptrs[] = {V, carry, carry2, ctl, flags, digits, errlog, qtwC, qtwR, qtwL, tw1, tw2, pos_of_c, wA, iwA, sA, wB, iwB, sB};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}

cudaError_t LargeTest::init(uint64_t p_, uint64_t n, int log_c, int rows_) {
    p = p_;
    N = n;
    M = N / 2;
    int mixed_log_c = 0;
    if (large_mixed_length_supported(N, &r0, &mixed_log_c)) {
        // R = R0 2^9 columns, rows of M / R (the row shape is fixed: no autotuned split here)
        logN = -1;
        logC = mixed_log_c;
        rows = large_rows_per_block(logC);
        if (!large_rows_supported(logC, rows)) return cudaErrorInvalidValue;
        C = 1 << logC;
        R = (int)(M / (uint64_t)C);
        logR = large_col_code(r0, 9);
    } else {
        r0 = 1;
        logN = 0;
        while ((1ull << logN) < N) ++logN;
        if ((1ull << logN) != N) return cudaErrorInvalidValue;
        logC = large_default_log_c(logN);
        if (log_c >= 0) logC = log_c;
        rows = rows_ ? rows_ : large_rows_per_block(logC);
        if (!large_split_supported(logN, logC, rows)) return cudaErrorInvalidValue;
        logR = logN - 1 - logC;
        C = 1 << logC;
        R = 1 << logR;
    }
    nblocks = R / rows;
    int log_m = 0;
    while ((1ull << log_m) < M) ++log_m;
    // four-step twiddles w_M^x, x = a c < M, as tw1[x mod 2^s] tw2[x >> s]
    const int s = std::max(logC, (log_m + 1) / 2);
    cudaError_t e;
    if ((e = configure_large(logC, rows, logR))) return e;
    // tables
    if ((e = upload(&qtwC, padded_full_table(C)))) return e;
    if (r0 == 1) {
        if ((e = upload(&qtwR, spread_quarter_table(R)))) return e;  // the column pass reads qpad_s
    } else {
        if ((e = upload(&qtwR, padded_quarter_table(R)))) return e;    // R = R0 2^9 (twiddle_r)
        if ((e = upload(&qtwL, padded_quarter_table(R / r0)))) return e;
    }
    if ((e = upload(&tw1, omega_table(M, 1ull << s, 1)))) return e;
    if ((e = upload(&tw2, omega_table(M, (M + (1ull << s) - 1) >> s, 1ull << s)))) return e;
    std::vector<int> pc(C);
    for (int c = 0; c < C; ++c) pc[c] = host_pos_of_freq(logC, large_row_log_e(logC, rows), c);
    if ((e = upload(&pos_of_c, pc))) return e;
    std::vector<double> hwA(2 * R), hiwA(2 * R), hwB(C), hiwB(C);
    std::vector<int> hsA(2 * R), hsB(C);
    const long double Nl = (long double)N;
    for (int j = 0; j < 2 * R; ++j) {
        const uint64_t sj = (N - (uint64_t)(((unsigned __int128)j * p) % N)) % N;
        hsA[j] = (int)sj;
        hwA[j] = (double)exp2l((long double)sj / Nl);
        hiwA[j] = (double)exp2l(-(long double)sj / Nl);
    }
    for (int b = 0; b < C; ++b) {
        const uint64_t sj = (N - (uint64_t)(((unsigned __int128)2 * R * b * p) % N)) % N;
        hsB[b] = (int)sj;
        hwB[b] = (double)exp2l((long double)sj / Nl);
        hiwB[b] = (double)(exp2l(-(long double)sj / Nl) / (4.0L * (long double)M));
    }
    if ((e = upload(&wA, hwA))) return e;
    if ((e = upload(&iwA, hiwA))) return e;
    if ((e = upload(&sA, hsA))) return e;
    if ((e = upload(&wB, hwB))) return e;
    if ((e = upload(&iwB, hiwB))) return e;
    if ((e = upload(&sB, hsB))) return e;
    // state
    if ((e = cudaMalloc(&V, M * sizeof(double2)))) return e;
    // carry slots and flags: one per tile plus slot 0 for the wrap-around job
    if ((e = cudaMalloc(&carry, (size_t)(nblocks + 1) * C * sizeof(double)))) return e;
    if ((e = cudaMalloc(&carry2, (size_t)(nblocks + 1) * C * sizeof(double)))) return e;
    if ((e = cudaMalloc(&ctl, sizeof(LargeCtl)))) return e;
    if ((e = cudaMemset(ctl, 0, sizeof(LargeCtl)))) return e;
    if ((e = cudaMalloc(&flags, (size_t)(nblocks + 1) * sizeof(unsigned)))) return e;
    if ((e = cudaMemset(flags, 0, (size_t)(nblocks + 1) * sizeof(unsigned)))) return e;
    if ((e = cudaMalloc(&digits, N * sizeof(int)))) return e;
    errlog_len = 1 << 16;
    if ((e = cudaMalloc(&errlog, errlog_len * sizeof(float)))) return e;
    if ((e = cudaMemset(errlog, 0, errlog_len * sizeof(float)))) return e;

    LargeArgs& A = args;
    std::memset(&A, 0, sizeof A);
    A.V = V;
    A.qtwC = qtwC;
    A.qtwR = qtwR;
    A.qtwL = qtwL;
    A.tw1 = tw1;
    A.tw2 = tw2;
    A.pos_of_c = pos_of_c;
    A.wA = wA;
    A.iwA = iwA;
    A.sA = sA;
    A.wB = wB;
    A.iwB = iwB;
    A.sB = sB;
    A.carry = carry;
    A.carry2 = carry2;
    A.ctl = ctl;
    A.flags = flags;
    A.digits = digits;
    A.errlog = errlog;
    A.errlog_len = errlog_len;
    A.spin_limit = kSpinLimit;
    A.dump = 0;
    A.tw_shift = s;
    A.C = C;
    A.R = R;
    A.nblocks = nblocks;
    A.q = (int)(p / N);
    A.rem = (int)(p % N);
    A.N = (int)N;
    A.logN = logN;
    return cudaSuccess;
}

cudaError_t LargeTest::start_seed(cudaStream_t st) {
    cudaError_t e = seed_digits_device(digits, N, st);
    return e ? e : start_device(st);
}

cudaError_t LargeTest::start_device(cudaStream_t st) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(ctl, 0, sizeof(LargeCtl), st))) return e;
    if ((e = cudaMemsetAsync(flags, 0, (size_t)(nblocks + 1) * sizeof(unsigned), st))) return e;
    if ((e = cudaMemsetAsync(errlog, 0, errlog_len * sizeof(float), st))) return e;
    if ((e = launch_large_row(logC, rows, LARGE_INIT, args, st))) return e;
    if ((e = launch_large_col(logR, args, st))) return e;
    done = 1;
    return cudaSuccess;
}

cudaError_t LargeTest::step_plain(uint64_t k, bool dump_last, cudaStream_t st) {
    cudaError_t e;
    for (uint64_t i = 0; i < k; ++i) {
        LargeArgs a = args;
        a.dump = (dump_last && i + 1 == k) ? 1 : 0;
        if ((e = launch_large_row(logC, rows, LARGE_ITER, a, st))) return e;
        if ((e = launch_large_col(logR, a, st))) return e;
    }
    done += k;
    return cudaSuccess;
}

// k squarings as replays of a captured graph of kGraphChunk (row, col) pairs plus a remainder.
cudaError_t LargeTest::step(uint64_t k, cudaStream_t st) {
    cudaError_t e;
    if (!exec && k >= (uint64_t)kGraphChunk) {
        cudaStream_t cap;
        if ((e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking))) return e;
        if ((e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal))) return e;
        for (int i = 0; i < kGraphChunk; ++i) {
            launch_large_row(logC, rows, LARGE_ITER, args, cap);
            launch_large_col(logR, args, cap);
        }
        cudaGraph_t g;
        e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (e) return e;
        e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (e) return e;
    }
    uint64_t left = k;
    while (exec && left >= (uint64_t)kGraphChunk) {
        if ((e = cudaGraphLaunch(exec, st))) return e;
        left -= kGraphChunk;
        done += kGraphChunk;
    }
    return step_plain(left, false, st);
}

cudaError_t LargeTest::final_pass(cudaStream_t st) {
    cudaError_t e;
    if ((e = launch_large_row(logC, rows, LARGE_FINAL, args, st))) return e;
    // the squarings may resume from this state at the same epoch: clear the flags FINAL set
    return cudaMemsetAsync(flags, 0, (size_t)(nblocks + 1) * sizeof(unsigned), st);
}

cudaError_t LargeTest::finish(cudaStream_t st, std::vector<int>& out) {
    cudaError_t e;
    if ((e = final_pass(st))) return e;
    out.resize(2 * M);
    if ((e = cudaMemcpyAsync(out.data(), digits, 2 * M * sizeof(int), cudaMemcpyDeviceToHost, st))) return e;
    return cudaStreamSynchronize(st);
}

cudaError_t LargeTest::diag_withhold_wrap(unsigned long long spin_limit, cudaStream_t st, bool& timed_out) {
    LargeCtl h;
    cudaError_t e = read_ctl(h, st);
    if (e) return e;
    // tickets start at 1: ticket 0, the wrap-around job, is never handed out, so tile 0 and the
    // last tile wait for its flag until their limit runs out; every index stays that of a tile
    const unsigned one = 1u;
    count_h2d(sizeof one);
    if ((e = cudaMemcpyAsync(&ctl->ticket[h.epoch & 1u], &one, sizeof one, cudaMemcpyHostToDevice, st))) return e;
    LargeArgs a = args;
    a.spin_limit = spin_limit;
    if ((e = launch_large_row(logC, rows, LARGE_ITER, a, st, nblocks))) return e;
    if ((e = read_ctl(h, st))) return e;
    timed_out = h.timeout != 0;
    return cudaSuccess;
}

cudaError_t LargeTest::read_ctl(LargeCtl& h, cudaStream_t st) {
    cudaError_t e = cudaMemcpyAsync(&h, ctl, sizeof(LargeCtl), cudaMemcpyDeviceToHost, st);
    if (e) return e;
    return cudaStreamSynchronize(st);
}

cudaError_t LargeTest::clear_err_since(cudaStream_t st) {
    return cudaMemsetAsync(&ctl->err_since, 0, sizeof(unsigned long long), st);
}

namespace {

// Launches k (row, column) pairs with an event after each launch; mean device us of each pass.
template <class Row, class Col>
cudaError_t time_pairs(uint64_t k, cudaStream_t st, Row row, Col col, double& row_us, double& col_us) {
    row_us = col_us = 0.0;
    if (k == 0) return cudaSuccess;
    std::vector<cudaEvent_t> ev(2 * k + 1, nullptr);
    cudaError_t e = cudaSuccess;
    for (auto& x : ev)
        if (!e) e = cudaEventCreate(&x);
    if (!e) e = cudaEventRecord(ev[0], st);
    for (uint64_t i = 0; i < k && !e; ++i) {
        e = row();
        if (!e) e = cudaEventRecord(ev[2 * i + 1], st);
        if (!e) e = col();
        if (!e) e = cudaEventRecord(ev[2 * i + 2], st);
    }
    if (!e) e = cudaEventSynchronize(ev.back());
    double r = 0.0, c = 0.0;
    for (uint64_t i = 0; i < k && !e; ++i) {
        float a = 0.f, b = 0.f;
        e = cudaEventElapsedTime(&a, ev[2 * i], ev[2 * i + 1]);
        if (!e) e = cudaEventElapsedTime(&b, ev[2 * i + 1], ev[2 * i + 2]);
        r += a;
        c += b;
    }
    for (auto& x : ev)
        if (x) cudaEventDestroy(x);
    row_us = 1e3 * r / (double)k;
    col_us = 1e3 * c / (double)k;
    return e;
}

}  // namespace

cudaError_t LargeTest::time_passes(uint64_t k, cudaStream_t st, double& row_us, double& col_us) {
    cudaError_t e = time_pairs(
        k, st, [&] { return launch_large_row(logC, rows, LARGE_ITER, args, st); },
        [&] { return launch_large_col(logR, args, st); }, row_us, col_us);
    if (!e) done += k;
    return e;
}

// The balanced digits of s_0 = 4 (digit 0 holds 4; every digit has >= 3 bits here), written on
// the device: zero, then the low byte of digit 0 set to 4 (int32, little-endian). No host buffer
// and no host-to-device copy of N zero digits.
cudaError_t seed_digits_device(int* digits, uint64_t n, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(digits, 0, (size_t)n * sizeof(int), st);
    if (!e) e = cudaMemsetAsync(digits, 4, 1, st);
    return e;
}

}  // namespace llg

// ---- two-pass NTT engine ----------------------------------------------------------------------

namespace llg {

namespace {

constexpr uint64_t kQ = 0xFFFFFFFF00000001ull;
uint64_t qmul(uint64_t a, uint64_t b) { return (uint64_t)(((unsigned __int128)a * b) % kQ); }
uint64_t qpow(uint64_t a, uint64_t e) {
    uint64_t r = 1;
    a %= kQ;
    while (e) {
        if (e & 1) r = qmul(r, a);
        a = qmul(a, a);
        e >>= 1;
    }
    return r;
}

int ntt_pos_of_freq(int log_l, int k) {  // SmallGeom<log_l> (16 values per thread) digit reversal
    const int L = 1 << log_l, P = (log_l + 3) / 4;
    const int RLAST = (log_l % 4 == 0) ? 16 : (1 << (log_l % 4));
    const int klast = k / (L / RLAST);
    int low = k % (L / RLAST), rest = 0;
    for (int q = 0; q < P - 1; ++q) {
        rest = (rest << 4) | (low & 15);
        low >>= 4;
    }
    return rest * RLAST + klast;
}

std::vector<uint64_t> ntt_half(int log_l) {  // w_L^r at gl::qpad8(r), r < L/2
    const uint32_t L = 1u << log_l, QL = L / 2;
    std::vector<uint64_t> t(QL + (QL >> 4) + 1, 0ull);
    const uint64_t w = qpow(7, (kQ - 1) / L);
    uint64_t x = 1;
    for (uint32_t r = 0; r < QL; ++r) {
        t[r + (r >> 4)] = x;
        x = qmul(x, w);
    }
    return t;
}

}  // namespace

bool ntt_host_constants(int log_n, uint64_t& omega, uint64_t& root2, uint64_t& inv_root2, uint64_t& invN) {
    // cuda/ll_ntt.cu:182-195: w_N = 7^((q-1)/N); an N-th root of 2 from a primitive (192N)-th root
    const uint64_t N = 1ull << log_n;
    omega = qpow(7, (kQ - 1) / N);
    const uint64_t om = qpow(7, (kQ - 1) / (192 * N)), r192 = qpow(om, N);
    uint64_t pw = 1, s = 0;
    for (; s < 192; ++s) {
        if (pw == 2) break;
        pw = qmul(pw, r192);
    }
    if (s == 192) return false;
    root2 = qpow(om, s);
    inv_root2 = qpow(root2, kQ - 2);
    invN = qpow(N % kQ, kQ - 2);
    return true;
}

bool ntt_large_length_supported(int log_n) { return log_n >= 14 && log_n <= 23; }

NttLargeTest::~NttLargeTest() {
    if (exec) cudaGraphExecDestroy(exec);
    for (int i = 0; i < nmem; ++i)
        if (mem[i]) cudaFree(mem[i]);
}

cudaError_t NttLargeTest::init(uint64_t p_, int log_n) {
    p = p_;
    logN = log_n;
    N = 1ull << logN;
    logC = std::min(10, std::max(7, logN / 2));
    logR = logN - logC;
    C = 1 << logC;
    R = 1 << logR;
    nblocks = R / 4;
    const int s = std::max(logC, (logN + 1) / 2);
    cudaError_t e;
    if ((e = configure_ntt_large(logC, logR))) return e;
    uint64_t omega, root2, iroot2, invN;
    if (!ntt_host_constants(logN, omega, root2, iroot2, invN)) return cudaErrorInvalidValue;
    auto up = [&](const auto& vec, const auto** dptr) -> cudaError_t {
        const size_t bytes = vec.size() * sizeof(vec[0]);
        void* d = nullptr;
        cudaError_t er = cudaMalloc(&d, bytes);
        if (er) return er;
        mem[nmem++] = d;
        *dptr = static_cast<decltype(vec.data())>(d);
        count_h2d(bytes);
        return cudaMemcpy(d, vec.data(), bytes, cudaMemcpyHostToDevice);
    };
    auto alloc = [&](size_t bytes, void** d) -> cudaError_t {
        cudaError_t er = cudaMalloc(d, bytes);
        if (!er) mem[nmem++] = *d;
        return er;
    };
    NttLargeArgs& A = args;
    std::memset(&A, 0, sizeof A);
    std::vector<uint64_t> qc = ntt_half(logC), qr = ntt_half(logR);
    std::vector<uint64_t> t1(1ull << s), t2(N >> s);
    {
        uint64_t x = 1;
        for (size_t i = 0; i < t1.size(); ++i) {
            t1[i] = x;
            x = qmul(x, omega);
        }
        const uint64_t st = qpow(omega, 1ull << s);
        x = 1;
        for (size_t i = 0; i < t2.size(); ++i) {
            t2[i] = x;
            x = qmul(x, st);
        }
    }
    std::vector<int> pc(C), hsA(R), hsB(C);
    for (int c = 0; c < C; ++c) pc[c] = ntt_pos_of_freq(logC, c);
    std::vector<uint64_t> hwA(R), hiwA(R), hwB(C), hiwB(C);
    for (int a = 0; a < R; ++a) {
        const uint64_t sj = (N - (uint64_t)(((unsigned __int128)a * p) % N)) % N;
        hsA[a] = (int)sj;
        hwA[a] = qpow(root2, sj);
        hiwA[a] = qpow(iroot2, sj);
    }
    for (int b = 0; b < C; ++b) {
        const uint64_t sj = (N - (uint64_t)(((unsigned __int128)R * b * p) % N)) % N;
        hsB[b] = (int)sj;
        hwB[b] = qpow(root2, sj);
        hiwB[b] = qmul(qpow(iroot2, sj), invN);
    }
    const uint64_t *cqc, *cqr, *ct1, *ct2, *cwA, *ciwA, *cwB, *ciwB;
    const int *cpc, *csA, *csB;
    if ((e = up(qc, &cqc)) || (e = up(qr, &cqr)) || (e = up(t1, &ct1)) || (e = up(t2, &ct2)) ||
        (e = up(pc, &cpc)) || (e = up(hwA, &cwA)) || (e = up(hiwA, &ciwA)) || (e = up(hsA, &csA)) ||
        (e = up(hwB, &cwB)) || (e = up(hiwB, &ciwB)) || (e = up(hsB, &csB)))
        return e;
    void *dV, *dc1, *dc2, *dc3, *dh, *dctl, *dd, *dfl;
    if ((e = alloc(N * sizeof(uint64_t), &dV)) || (e = alloc((size_t)nblocks * C * sizeof(long long), &dc1)) ||
        (e = alloc((size_t)nblocks * C * sizeof(int), &dc2)) || (e = alloc((size_t)nblocks * C * sizeof(int), &dc3)) ||
        (e = alloc((size_t)C * (sizeof(long long) + 2 * sizeof(int)), &dh)) ||
        (e = alloc(sizeof(LargeCtl), &dctl)) || (e = alloc(N * sizeof(int), &dd)) ||
        (e = alloc((size_t)nblocks * sizeof(unsigned), &dfl)))
        return e;
    if ((e = cudaMemset(dctl, 0, sizeof(LargeCtl)))) return e;
    if ((e = cudaMemset(dfl, 0, (size_t)nblocks * sizeof(unsigned)))) return e;
    ctl = static_cast<LargeCtl*>(dctl);
    digits = static_cast<int*>(dd);
    A.V = static_cast<uint64_t*>(dV);
    A.qtwC = cqc;
    A.qtwR = cqr;
    A.tw1 = ct1;
    A.tw2 = ct2;
    A.pos_of_c = cpc;
    A.wA = cwA;
    A.iwA = ciwA;
    A.sA = csA;
    A.wB = cwB;
    A.iwB = ciwB;
    A.sB = csB;
    A.c1 = static_cast<long long*>(dc1);
    A.c2 = static_cast<int*>(dc2);
    A.c3 = static_cast<int*>(dc3);
    A.halo = static_cast<long long*>(dh);
    A.ctl = ctl;
    A.flags = static_cast<unsigned*>(dfl);
    A.digits = digits;
    A.dump = 0;
    A.tw_shift = s;
    A.C = C;
    A.R = R;
    A.nblocks = nblocks;
    A.q = (int)(p >> logN);
    A.rem = (int)(p & (N - 1));
    A.logN = logN;
    return cudaSuccess;
}

cudaError_t NttLargeTest::start_seed(cudaStream_t st) {
    cudaError_t e = seed_digits_device(digits, N, st);
    return e ? e : start_device(st);
}

cudaError_t NttLargeTest::start_device(cudaStream_t st) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(ctl, 0, sizeof(LargeCtl), st))) return e;
    if ((e = cudaMemsetAsync(args.flags, 0, (size_t)nblocks * sizeof(unsigned), st))) return e;
    if ((e = launch_ntt_row(logC, LARGE_INIT, args, st))) return e;
    if ((e = launch_ntt_col(logR, args, st))) return e;
    done = 1;
    return cudaSuccess;
}

cudaError_t NttLargeTest::step(uint64_t k, cudaStream_t st) {
    cudaError_t e;
    if (!exec && k >= (uint64_t)kGraphChunk) {
        cudaStream_t cap;
        if ((e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking))) return e;
        if ((e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal))) return e;
        for (int i = 0; i < kGraphChunk; ++i) {
            launch_ntt_row(logC, LARGE_ITER, args, cap);
            launch_ntt_col(logR, args, cap);
        }
        cudaGraph_t g;
        e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (e) return e;
        e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (e) return e;
    }
    uint64_t left = k;
    while (exec && left >= (uint64_t)kGraphChunk) {
        if ((e = cudaGraphLaunch(exec, st))) return e;
        left -= kGraphChunk;
        done += kGraphChunk;
    }
    for (uint64_t i = 0; i < left; ++i) {
        if ((e = launch_ntt_row(logC, LARGE_ITER, args, st))) return e;
        if ((e = launch_ntt_col(logR, args, st))) return e;
    }
    done += left;
    return cudaSuccess;
}

cudaError_t NttLargeTest::final_pass(cudaStream_t st) {
    cudaError_t e;
    if ((e = launch_ntt_row(logC, LARGE_FINAL, args, st))) return e;
    if ((e = cudaMemsetAsync(&ctl->halo_read, 0, sizeof(unsigned), st))) return e;
    return cudaMemsetAsync(args.flags, 0, (size_t)nblocks * sizeof(unsigned), st);
}

cudaError_t NttLargeTest::finish(cudaStream_t st, std::vector<int>& out) {
    cudaError_t e;
    if ((e = final_pass(st))) return e;
    out.resize(N);
    if ((e = cudaMemcpyAsync(out.data(), digits, N * sizeof(int), cudaMemcpyDeviceToHost, st))) return e;
    return cudaStreamSynchronize(st);
}

cudaError_t NttLargeTest::time_passes(uint64_t k, cudaStream_t st, double& row_us, double& col_us) {
    cudaError_t e = time_pairs(
        k, st, [&] { return launch_ntt_row(logC, LARGE_ITER, args, st); },
        [&] { return launch_ntt_col(logR, args, st); }, row_us, col_us);
    if (!e) done += k;
    return e;
}

cudaError_t NttLargeTest::read_ctl(LargeCtl& h, cudaStream_t st) {
    cudaError_t e = cudaMemcpyAsync(&h, ctl, sizeof(LargeCtl), cudaMemcpyDeviceToHost, st);
    if (e) return e;
    return cudaStreamSynchronize(st);
}

}  // namespace llg
