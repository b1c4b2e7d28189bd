/* llgpu: B200 (sm_100a) Lucas-Lehmer squaring engine -- the C-ABI drop-in boundary.
 *
 * Plain C types only (no CUDA or torch types): pointers, sizes, status codes. Every function is
 * callable from many host threads at once; each host thread gets its own CUDA stream and device
 * buffers. All results are exact: floating-point runs whose round-off ever exceeds the abort
 * threshold are redone at a longer transform on the GPU (no CPU fallback).
 *
 * Each entry point names the reference interface it replaces (wadeghcp/MersennePrime_Python_CPP_
 * GMP_BenchMark; file:line). The reference binds those functions to Python with pybind11
 * (lucaslehmer.cpp:344-387, cuda/ll_ntt.cu:274-281); this library's pybind11 modules
 * (lucaslehmer, lucaslehmer_cuda) bind these entry points the same way.
 */
#ifndef LLGPU_H
#define LLGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LLG_ABI_VERSION 1

/* Status codes (return values and llg_result.status). */
enum {
    LLG_OK = 0,
    LLG_E_CUDA = 1,        /* a CUDA runtime call failed (message: llg_last_error()) */
    LLG_E_NODEV = 2,       /* no CUDA device visible */
    LLG_E_ARG = 3,         /* invalid argument (null pointer, size too small, bad engine) */
    LLG_E_UNSUPPORTED = 4, /* exponent / length outside what the engine handles */
    LLG_E_ROUNDOFF = 5,    /* round-off stayed above the threshold at every length tried */
    LLG_E_TIMEOUT = 6,     /* a bounded device-side wait gave up */
    LLG_E_NOMEM = 7        /* device allocation failed */
};

/* Engines. FP64 = Crandall-Fagin IBDWT in double precision (lucaslehmer.cpp:209-342);
 * NTT = the same digit layout in GF(2^64 - 2^32 + 1), exact (cuda/ll_ntt.cu). */
enum { LLG_ENGINE_FP64 = 0, LLG_ENGINE_NTT = 1 };

typedef struct llg_result {
    uint64_t p;
    uint64_t iters;       /* squarings performed: p-2, or the requested interim count */
    uint64_t res64;       /* low 64 bits of s_iters mod 2^p - 1, in [0, 2^p - 1) */
    double max_err;       /* worst |x - round(x)| over the run (FP64; 0 for NTT) */
    double seconds;       /* device time of the test */
    uint32_t n;           /* transform length that produced the result */
    uint32_t escalations; /* times the length was raised after a round-off abort */
    int32_t is_zero;      /* residue == 0; for a full run: 2^p - 1 is prime */
    int32_t status;       /* LLG_OK or an LLG_E_* code for this exponent */
} llg_result;

/* Human-readable text of a status code; llg_last_error(): detail of this thread's last failure. */
const char* llg_status_string(int status);
const char* llg_last_error(void);

/* (name, SM count, global memory) of the current device.
 * Replaces device_info(), cuda/ll_ntt.cu:269-272. */
int llg_device_info(char* name, size_t name_cap, int* sms, uint64_t* total_mem);

/* Transform length the FP64 engine uses for p at <= max_bpw bits per digit (<= 0: the module
 * default, see llg_set_max_bpw); 0 = p outside the engine's range.
 * Replaces fft_length(), lucaslehmer.cpp:244-254. */
uint32_t llg_fft_length(uint64_t p, double max_bpw);
/* Default bits-per-digit bound of llg_fft_length (18 unless changed).
 * Replaces set_fft_bits_per_word(), lucaslehmer.cpp:368 (g_max_bpw, lucaslehmer.cpp:246). */
int llg_set_max_bpw(double bpw);
double llg_get_max_bpw(void);
/* Round-off bound of the FP64 engine (default 0.4, in (0, 0.5)): a test whose worst
 * |x - round(x)| exceeds it is redone at a longer length (two-pass lengths: from the residue of
 * the last check that stayed within it). Replaces the fixed 0.35 bound of lucaslehmer.cpp:296. */
int llg_set_roundoff_limit(double limit);
double llg_get_roundoff_limit(void);
/* NTT length for p (exactness bound ceil(p/N) <= (63 - log2 N)/2); 0 = cannot take.
 * Replaces ntt_length(), cuda/ll_ntt.cu:172-180. */
uint32_t llg_ntt_length(uint64_t p);
/* Shape of the two-pass FP64 engine at N = 2^log_n (2^14 .. 2^23): rows of 2^log_c complex
 * values, columns of 2^(log_n - 1 - log_c), `rows` rows per row-pass block (2 or 4; 0: the
 * default for log_c). Tests created afterwards use it; log_c < 0 restores the built-in shape. The
 * autotuner (llgpu.autotune) times the supported shapes and sets the fastest. No reference
 * counterpart (FFTW_MEASURE planning, lucaslehmer.cpp:232-242, is the nearest).
 * llg_get_large_split returns the row length in force (-1 for a length without one) and its rows
 * per block in *rows (may be null). */
int llg_set_large_split(int log_n, int log_c, int rows);
int llg_get_large_split(int log_n, int* rows);
/* Length choice for whole-test exponents: where the bits-per-digit rule of llg_fft_length gives
 * the whole-test length n_rule, use n_use (>= n_rule; 0 or n_rule: the rule's own) for exponents it
 * is usable for. The range autotuner (llgpu.autotune_range) times the candidates per length and
 * sets the fastest; the tune file of llg_set_large_split also keeps these. No reference counterpart
 * (the reference always takes the smallest {1,3,5} x 2^k length, lucaslehmer.cpp:244-254).
 * llg_get_length_choice returns the length used where the rule gives n_rule. */
int llg_set_length_choice(uint32_t n_rule, uint32_t n_use);
uint32_t llg_get_length_choice(uint32_t n_rule);
/* Largest exponent an engine handles. Replaces max_exponent(), cuda/ll_ntt.cu:279. */
uint64_t llg_max_exponent(int engine);

/* One Lucas-Lehmer test (max_iters == 0) or its first max_iters squarings, on the GPU.
 * n == 0 picks the length (llg_fft_length / llg_ntt_length). words (optional, nwords >=
 * ceil(p/64)): the full residue s_iters mod 2^p - 1, little-endian 64-bit limbs.
 * Replaces lucas_lehmer_fft_raw() + the GMP rebuild, lucaslehmer.cpp:257-329, and, for the exact
 * engine, lucas_lehmer_n(), lucaslehmer.cpp:29-58. */
int llg_run(uint64_t p, uint64_t max_iters, int engine, uint32_t n, llg_result* out,
            uint64_t* words, size_t nwords);

/* Many exponents in one call: grouped by transform length, one batched launch per group, the
 * groups running concurrently. out[i] corresponds to ps[i]. words_out (optional): for each i,
 * ceil(ps[i]/64) limbs, concatenated in input order.
 * Replaces lucas_lehmer_batch() / run_batch(), cuda/ll_ntt.cu:198-267. */
int llg_run_batch(const uint64_t* ps, size_t count, uint64_t max_iters, int engine,
                  llg_result* out, uint64_t* words_out, size_t words_cap);

/* Device-resident batches: the same work as llg_run_batch split into create (upload the job
 * lists, allocate), launch (enqueue every length group on its own stream, forked from and joined
 * back into `stream`, so events recorded on `stream` bracket the whole batch; stream == NULL uses
 * a per-thread stream) and results (wait, read back, redo round-off aborts at longer lengths,
 * rebuild residues). A batch may be launched again after its results are read.
 * flags: LLG_BATCH_KEEP_WORDS keeps full residues for llg_batch_results; LLG_BATCH_ERRLOG keeps
 * the per-iteration max round-off of a single-exponent batch for llg_batch_errlog.
 * Replaces run_batch()'s upload / launch / readback phases, cuda/ll_ntt.cu:213-235. */
typedef struct llg_batch llg_batch;
#define LLG_BATCH_KEEP_WORDS 1
#define LLG_BATCH_ERRLOG 2
int llg_batch_create(const uint64_t* ps, size_t count, uint64_t max_iters, int engine, int flags,
                     llg_batch** out);
int llg_batch_launch(llg_batch* b, void* stream);
int llg_batch_results(llg_batch* b, llg_result* out, uint64_t* words, size_t words_cap);
int llg_batch_errlog(llg_batch* b, float* log, size_t cap, size_t* len);
/* Device time of the last launch: CUDA events recorded on the launch stream before the fork and
 * after the join (waits for the launch to finish). */
int llg_batch_device_ms(llg_batch* b, float* ms);
void llg_batch_destroy(llg_batch* b);

/* One exponent's device state on a two-pass engine (FP64 or NTT, lengths 2^14 .. 2^23), for callers that
 * drive the iterations themselves (interim residues, timing on their own stream):
 * create (tables, state; n == 0 picks the length), start (s_0 = 4 and the first squaring),
 * iterate (enqueue squarings as CUDA-graph replays, no host sync), read (final row pass, digits
 * back, exact residue; waits; the squarings may resume after it). llg_result.iters counts the
 * squarings done since s_0 (start's included);
 * llg_result.status is LLG_E_ROUNDOFF when the worst round-off exceeded 0.4 (no escalation here).
 * llg_test_errlog (FP64): per-squaring max round-off (ring of 65536 entries; entry e is squaring
 * e, from 1); it waits for the device first.
 * Replaces the iteration loop of lucas_lehmer_fft_raw(), lucaslehmer.cpp:281-311, for large p. */
typedef struct llg_test llg_test;
int llg_test_create(uint64_t p, uint32_t n, int engine, llg_test** out);
int llg_test_start(llg_test* t, void* stream);
int llg_test_iterate(llg_test* t, uint64_t iters, void* stream);
int llg_test_read(llg_test* t, void* stream, llg_result* out, uint64_t* words, size_t nwords);
int llg_test_errlog(llg_test* t, float* log, size_t cap, size_t* len);
/* Sets the test's state to a residue s (ceil(p/64) little-endian limbs, s < 2^p) reached after
 * `iters_done` squarings and starts the next squaring, as llg_test_start does from s_0 = 4. The
 * digits are formed on the GPU at the test's own length, so a residue from any length (or from
 * another engine) resumes here; llg_test_read's words are such a residue. Replaces restarting
 * lucas_lehmer_fft_raw() from s_0 (lucaslehmer.cpp:272-273) after a round-off abort
 * (lucaslehmer.cpp:296, 334): a test moved to a longer length goes on from its last residue. */
int llg_test_load(llg_test* t, const uint64_t* words, size_t nwords, uint64_t iters_done, void* stream);
/* Diagnostic of the bounded waits (FP64 engine): one row pass whose wrap-around job is withheld
 * and whose flag waits give up after spin_limit sleeps of ~64 ns. Tile 0 and the last tile wait
 * for that job's flag, give up, and the kernel returns; the call then reports LLG_E_TIMEOUT.
 * The test's state is invalid afterwards (destroy it). No reference counterpart. */
int llg_test_diag_withhold_wrap(llg_test* t, uint64_t spin_limit, void* stream);
/* `iters` more squarings launched one pass at a time with CUDA events between the launches (no
 * graph): the mean device time in microseconds of the row pass and of the column pass. Waits. */
int llg_test_time_passes(llg_test* t, uint64_t iters, void* stream, double* row_us, double* col_us);
void llg_test_destroy(llg_test* t);

/* Exact residue of balanced (or any signed) digits: s = sum_j d_j 2^ceil(jp/n) mod 2^p - 1.
 * Host-only; needs no GPU. Replaces the GMP rebuild, lucaslehmer.cpp:312-323 and
 * cuda/ll_ntt.cu:238-252. Returns LLG_OK; *is_zero set when s == 0. */
int llg_residue_from_digits(uint64_t p, uint32_t n, const int64_t* digits, uint64_t* words,
                            size_t nwords, uint64_t* res64, int32_t* is_zero);

/* The same residue from digits already on the device (int32, natural order, as the two-pass
 * engine's final pass and llg_run_noalloc leave them), rebuilt on the GPU: word sums, a scan of the
 * +-1 carry chains, the fold of the bits above p into bit 0, the canonical zero. d_words (device,
 * ceil(p/64) words) may be null when only res64 / is_zero are wanted. Waits on `stream`.
 * Replaces the same GMP rebuild without copying the digits back. */
int llg_residue_from_digits_device(uint64_t p, uint32_t n, const int32_t* d_digits, uint64_t* d_words,
                                   uint64_t* res64, int32_t* is_zero, void* stream);

/* The two-pass engine for transform lengths 16,384 .. 65,536 without allocating device memory.
 * No counterpart in the reference: it serves callers that cannot call cudaMalloc (a host
 * framework that owns every device allocation through its own pool, or code that must not risk
 * the device-wide synchronisation cudaFree can cause while other work is in flight). All state
 * and tables live in one fixed device array of LLG_NOALLOC_SCRATCH_BYTES inside this library,
 * which every GPU that loads the library keeps until the process exits.
 * n must be a power of two in [16384, LLG_NOALLOC_MAX_N] usable for p (else LLG_E_UNSUPPORTED);
 * iters >= 1 squarings from s_0 = 4. digits_out: caller-owned DEVICE buffer of n int32 that
 * receives the balanced digits of s_iters in natural order (llg_residue_from_digits gives the
 * residue). max_err (host, optional): worst round-off. Enqueues on `stream` (NULL: legacy
 * default stream) and returns when it has finished; LLG_E_ROUNDOFF if the round-off exceeded 0.4.
 * Every call reuses the same array and leaves its contents behind; the call zeroes what has to
 * start at zero. Calls whose GPU work overlaps race on the array: serialise them. The first call
 * on each device looks up the array's device address. Every call uploads its tables with a
 * host-synchronous copy (skipped when p and n repeat the previous call's) and waits for `stream`,
 * so no call may be made while `stream` is being captured. A failure after work was enqueued
 * waits for `stream` too, so the array is idle when the call returns. */
#define LLG_NOALLOC_MAX_N 65536u
#define LLG_NOALLOC_SCRATCH_BYTES (640u * 1024u)
int llg_run_noalloc(uint64_t p, uint64_t iters, uint32_t n, int32_t* digits_out, double* max_err,
                    void* stream);

/* Roofline denominators measured on the current device: which = 0 FP64 FMA flops/s,
 * which = 1 INT32 multiply-adds/s (dependent chains on every SM). Diagnostic; no reference
 * counterpart. */
int llg_measure_peak(int which, double* ops_per_s);

/* Frees the two-pass test that llg_run keeps, with its tables, buffers and graphs, after a
 * single-exponent call (one per engine, for the next call on the same exponent, length and split
 * on the same device). Idle memory of up to ~30 bytes a digit is otherwise held until then. */
void llg_release_cached(void);

/* Bytes the library has copied from host to device since it was loaded, all threads together
 * (tables, job lists, residues handed in). Read before and after a call to count that call's
 * uploads. Diagnostic; no reference counterpart. */
uint64_t llg_h2d_bytes(void);

#ifdef __cplusplus
}
#endif

#endif
