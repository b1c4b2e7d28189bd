// llg_run_noalloc: the two-pass engine for lengths up to 65,536 without any device allocation.
//
// Why it exists: some callers cannot call cudaMalloc -- for example code running inside a host
// framework that owns every device allocation through its own pool, or a caller that must not
// trigger the implicit device synchronisation cudaFree can cause while other work is in flight.
// Every other entry point of this library allocates its state (the residue, the carry buffers,
// the control block, the twiddle and weight tables) per call or per test object. This one keeps
// all of that in one fixed-size array in device memory, declared below at file scope, which every
// GPU that loads this library holds until the process exits (kNoAllocScratchBytes bytes).
//
// Rules a caller must know:
//   * N (the transform length) must be a power of two from 16,384 to 65,536 and usable for p
//     (the same bits-per-digit rule as the allocating two-pass entry points); anything larger is
//     rejected with LLG_E_UNSUPPORTED because its state would not fit the array.
//   * All calls share the one array and it keeps the previous call's contents. The call clears
//     what must start at zero (the control block) and overwrites everything else before reading
//     it. Two calls whose GPU work overlaps (different streams, or different host threads) race on
//     the array and produce wrong results: serialise them.
//   * The first call on each device looks up the array's device address (cudaGetSymbolAddress).
//     Every call uploads its tables with a host-synchronous copy and waits for `stream` before it
//     returns, so no call may be made while `stream` is being captured into a CUDA graph.
//   * On an error after the first enqueue the call waits for `stream` before it returns, so the
//     array is idle again when the next call starts.
//   * The caller passes the output: digits_out, a device buffer of N int32 values, receives the
//     balanced digits of s_iters in natural order (llg_residue_from_digits turns them into the
//     residue). The call enqueues on `stream` (NULL: the legacy default stream) and returns after
//     that stream has finished.
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/llgpu.h"
#include "llg_device.cuh"
#include "llg_host.h"
#include "llg_internal.h"

namespace llg {

namespace {

constexpr size_t kNoAllocScratchBytes = 640u * 1024u;  // covers N = 65,536 (about 603 KiB used)
constexpr int kNoAllocMaxLog = 16;
constexpr int kMaxDevices = 64;

// The scratch itself. In host code this name is only a stand-in for the device copy: its device
// address comes from cudaGetSymbolAddress (per device) and only that address is given to kernels.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mx;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Host staging for the tables (no host allocation either): the largest table set is ~24 KiB. The
// tables are laid out contiguously in the array (qtwC .. sB), so one copy moves all of them.
constexpr size_t kStageBytes = 64u * 1024u;
alignas(256) unsigned char g_stage[kStageBytes];
// (p, n) whose tables the array holds, per device: a repeated call skips the upload
struct TableKey {
    uint64_t p = 0;
    uint32_t n = 0;
};
TableKey g_tables_for[kMaxDevices];

struct Layout {
    size_t V, carry, carry2, ctl, flags, qtwC, qtwR, tw1, tw2, pos_of_c, wA, iwA, sA, wB, iwB, sB, end;
};

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

// Rows per row-pass tile: 8 (the fewest tiles, so the fewest carry slots in the array).
constexpr int kTileRows = 8;

Layout layout(int logN, int logC, int logR, int s) {
    const size_t M = (size_t)1 << (logN - 1), C = (size_t)1 << logC, R = (size_t)1 << logR;
    const size_t nblocks = R / kTileRows;
    Layout L;
    size_t o = 0;
    L.V = o; o = up256(o + M * sizeof(double2));
    L.carry = o; o = up256(o + (nblocks + 1) * C * sizeof(double));  // slot 0: the wrap-around job
    L.carry2 = o; o = up256(o + (nblocks + 1) * C * sizeof(double));
    L.ctl = o; o = up256(o + sizeof(LargeCtl));
    L.flags = o; o = up256(o + (nblocks + 1) * sizeof(unsigned));
    L.qtwC = o; o = up256(o + qpad_len((uint32_t)C) * sizeof(double2));
    L.qtwR = o; o = up256(o + qpad_s_len((uint32_t)(R / 4)) * sizeof(double2));  // spread layout
    L.tw1 = o; o = up256(o + ((size_t)1 << s) * sizeof(double2));
    L.tw2 = o; o = up256(o + (M >> s) * sizeof(double2));
    L.pos_of_c = o; o = up256(o + C * sizeof(int));
    L.wA = o; o = up256(o + 2 * R * sizeof(double));
    L.iwA = o; o = up256(o + 2 * R * sizeof(double));
    L.sA = o; o = up256(o + 2 * R * sizeof(int));
    L.wB = o; o = up256(o + C * sizeof(double));
    L.iwB = o; o = up256(o + C * sizeof(double));
    L.sB = o; o = up256(o + C * sizeof(int));
    L.end = o;
    return L;
}

int pos_of_freq_host(int log_l, int k) {
    // digit reversal of the row FFT's output positions (radix 2^LE passes, the last one RLAST):
    // host copy of pos_of_freq for SmallGeom<log_l, LE>, LE as the row kernel is built
    const int LE = large_row_log_e(log_l, kTileRows), E = 1 << LE;
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

// Writes `count` table entries produced by f(i) into the host stage at byte offset `off`.
template <class T, class F>
void stage_table(size_t off, size_t count, F f) {
    T* dst = reinterpret_cast<T*>(g_stage + off);
    for (size_t i = 0; i < count; ++i) dst[i] = f(i);
}

int cuda_fail(const char* what, cudaError_t e) {
    char msg[256];
    snprintf(msg, sizeof msg, "llg_run_noalloc: %s: %s", what, cudaGetErrorString(e));
    return set_error(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? LLG_E_NODEV : LLG_E_CUDA, msg);
}

double2 omega(uint64_t period, uint64_t e) {
    const long double two_pi = 6.283185307179586476925286766559005768L;
    const long double ang = two_pi * (long double)(e % period) / (long double)period;
    return make_double2((double)cosl(ang), -(double)sinl(ang));
}

}  // namespace

}  // namespace llg

using namespace llg;

extern "C" int llg_run_noalloc(uint64_t p, uint64_t iters, uint32_t n, int32_t* digits_out,
                               double* max_err, void* stream) {
    if (!digits_out) return set_error(LLG_E_ARG, "llg_run_noalloc: digits_out is null");
    if (p < 3 || p % 2 == 0 || iters == 0)
        return set_error(LLG_E_ARG, "llg_run_noalloc: p must be odd and >= 3, iters >= 1");
    int logN = 0;
    while ((1ull << logN) < n) ++logN;
    if ((1ull << logN) != n || logN < 14 || logN > kNoAllocMaxLog)
        return set_error(LLG_E_UNSUPPORTED,
                         "llg_run_noalloc: n must be a power of two from 16384 to 65536 (its fixed "
                         "640 KiB device array holds nothing larger)");
    const uint64_t N = n, M = N / 2;
    // same usability rule as the allocating two-pass path: at least log2(N)/4 + 3 bits per digit
    if (4 * (p / N) < (uint64_t)logN + 12 || (p + N - 1) / N > 28)
        return set_error(LLG_E_UNSUPPORTED, "llg_run_noalloc: length not usable for this p (bits per digit)");
    const int logC = (logN <= 15) ? logN - 8 : 8;
    const int logR = logN - 1 - logC;
    const int C = 1 << logC, R = 1 << logR;
    const int s = logC > (logN / 2) ? logC : (logN / 2);
    const Layout L = layout(logN, logC, logR, s);
    if (L.end > kNoAllocScratchBytes) return set_error(LLG_E_UNSUPPORTED, "llg_run_noalloc: state exceeds the array");

    if (L.end - L.qtwC > kStageBytes) return set_error(LLG_E_UNSUPPORTED, "llg_run_noalloc: tables exceed the host stage");

    std::lock_guard<std::mutex> lk(g_noalloc_mx);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail("no current device", e);
    if (dev < 0 || dev >= kMaxDevices) return set_error(LLG_E_NODEV, "llg_run_noalloc: device ordinal out of range");
    if (!g_scratch_addr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) return cuda_fail("looking up the array's device address", e);
        g_scratch_addr[dev] = static_cast<unsigned char*>(ptr);
    }
    unsigned char* base = g_scratch_addr[dev];
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    e = configure_large(logC, kTileRows, logR);
    if (e != cudaSuccess) return cuda_fail("configuring the kernels", e);

    // tables (exact integers and long-double rounded values, as the allocating path uses), built
    // in the host stage at their offsets in the array and uploaded in one copy
    if (g_tables_for[dev].p != p || g_tables_for[dev].n != n) {
        g_tables_for[dev] = TableKey{};  // invalid until the upload below has completed
        const long double Nl = (long double)N;
        const size_t o = L.qtwC;
        std::memset(g_stage, 0, L.end - o);
        stage_table<double2>(L.qtwC - o, qpad_len((uint32_t)C), [&](size_t i) { return padded_quarter_slot(C, i); });
        {  // the column pass's quarter table in the spread layout: entry r at qpad_s(r)
            double2* q = reinterpret_cast<double2*>(g_stage + (L.qtwR - o));
            for (uint32_t r = 0; r < (uint32_t)R / 4; ++r) q[qpad_s(r)] = padded_quarter_slot(R, qpad(r));
        }
        stage_table<double2>(L.tw1 - o, (size_t)1 << s, [&](size_t i) { return omega(M, i); });
        stage_table<double2>(L.tw2 - o, (size_t)(M >> s), [&](size_t i) { return omega(M, (uint64_t)i << s); });
        stage_table<int>(L.pos_of_c - o, (size_t)C, [&](size_t i) { return pos_of_freq_host(logC, (int)i); });
        auto sAj = [&](size_t j) { return (N - (uint64_t)(((unsigned __int128)j * p) % N)) % N; };
        auto sBb = [&](size_t b) { return (N - (uint64_t)(((unsigned __int128)2 * R * b * p) % N)) % N; };
        stage_table<double>(L.wA - o, (size_t)2 * R, [&](size_t i) { return (double)exp2l((long double)sAj(i) / Nl); });
        stage_table<double>(L.iwA - o, (size_t)2 * R, [&](size_t i) { return (double)exp2l(-(long double)sAj(i) / Nl); });
        stage_table<int>(L.sA - o, (size_t)2 * R, [&](size_t i) { return (int)sAj(i); });
        stage_table<double>(L.wB - o, (size_t)C, [&](size_t i) { return (double)exp2l((long double)sBb(i) / Nl); });
        stage_table<double>(L.iwB - o, (size_t)C,
                            [&](size_t i) { return (double)(exp2l(-(long double)sBb(i) / Nl) / (4.0L * (long double)M)); });
        stage_table<int>(L.sB - o, (size_t)C, [&](size_t i) { return (int)sBb(i); });
        // pageable source: the copy has consumed the stage once the stream has finished it
        e = cudaMemcpyAsync(base + o, g_stage, L.end - o, cudaMemcpyHostToDevice, st);
        count_h2d(L.end - o);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            cudaStreamSynchronize(st);
            return cuda_fail("uploading the tables", e);
        }
        g_tables_for[dev] = TableKey{p, n};
    }

    LargeArgs A;
    std::memset(&A, 0, sizeof A);
    A.V = reinterpret_cast<double2*>(base + L.V);
    A.qtwC = reinterpret_cast<const double2*>(base + L.qtwC);
    A.qtwR = reinterpret_cast<const double2*>(base + L.qtwR);
    A.tw1 = reinterpret_cast<const double2*>(base + L.tw1);
    A.tw2 = reinterpret_cast<const double2*>(base + L.tw2);
    A.pos_of_c = reinterpret_cast<const int*>(base + L.pos_of_c);
    A.wA = reinterpret_cast<const double*>(base + L.wA);
    A.iwA = reinterpret_cast<const double*>(base + L.iwA);
    A.sA = reinterpret_cast<const int*>(base + L.sA);
    A.wB = reinterpret_cast<const double*>(base + L.wB);
    A.iwB = reinterpret_cast<const double*>(base + L.iwB);
    A.sB = reinterpret_cast<const int*>(base + L.sB);
    A.carry = reinterpret_cast<double*>(base + L.carry);
    A.carry2 = reinterpret_cast<double*>(base + L.carry2);
    A.ctl = reinterpret_cast<LargeCtl*>(base + L.ctl);
    A.flags = reinterpret_cast<unsigned*>(base + L.flags);
    A.digits = digits_out;
    A.errlog = nullptr;
    A.errlog_len = 1;
    A.spin_limit = kSpinLimit;
    A.dump = 0;
    A.tw_shift = s;
    A.C = C;
    A.R = R;
    A.nblocks = R / kTileRows;
    A.q = (int)(p >> logN);
    A.rem = (int)(p & (N - 1));
    A.N = (int)N;
    A.logN = logN;

    // s_0 = 4 as digits (the output buffer doubles as the INIT input), control block cleared.
    // From the first enqueue on, a failure waits for the stream before returning.
    auto fail_enqueued = [&](const char* what, cudaError_t err) {
        cudaStreamSynchronize(st);
        return cuda_fail(what, err);
    };
    static const int32_t four = 4;
    if ((e = cudaMemsetAsync(digits_out, 0, N * sizeof(int32_t), st)) != cudaSuccess)
        return fail_enqueued("clearing digits_out", e);
    count_h2d(sizeof four);
    if ((e = cudaMemcpyAsync(digits_out, &four, sizeof four, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return fail_enqueued("writing s_0", e);
    if ((e = cudaMemsetAsync(A.ctl, 0, sizeof(LargeCtl), st)) != cudaSuccess) return fail_enqueued("clearing the control block", e);
    if ((e = cudaMemsetAsync(A.flags, 0, (size_t)(A.nblocks + 1) * sizeof(unsigned), st)) != cudaSuccess)
        return fail_enqueued("clearing the carry flags", e);
    const int G = kTileRows;
    if ((e = launch_large_row(logC, G, LARGE_INIT, A, st)) != cudaSuccess) return fail_enqueued("row pass launch", e);
    if ((e = launch_large_col(logR, A, st)) != cudaSuccess) return fail_enqueued("column pass launch", e);
    for (uint64_t k = 1; k < iters; ++k) {
        if ((e = launch_large_row(logC, G, LARGE_ITER, A, st)) != cudaSuccess) return fail_enqueued("row pass launch", e);
        if ((e = launch_large_col(logR, A, st)) != cudaSuccess) return fail_enqueued("column pass launch", e);
    }
    if ((e = launch_large_row(logC, G, LARGE_FINAL, A, st)) != cudaSuccess) return fail_enqueued("row pass launch", e);
    LargeCtl h;
    if ((e = cudaMemcpyAsync(&h, A.ctl, sizeof(LargeCtl), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return fail_enqueued("reading the control block", e);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail("running the squarings", e);
    double err;
    std::memcpy(&err, &h.err_max, sizeof err);
    if (max_err) *max_err = err;
    if (h.timeout) return set_error(LLG_E_TIMEOUT, "llg_run_noalloc: a carry wait timed out");
    if (err > 0.4) return set_error(LLG_E_ROUNDOFF, "llg_run_noalloc: round-off above 0.4 at this length");
    return LLG_OK;
}
