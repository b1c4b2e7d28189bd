"""ctypes binding of the C-ABI in include/llgpu.h (libllgpu.so, built in-tree).

This is the reference-side binding a Python caller would add for the boundary (the pybind11
modules in this package bind the same entry points for the reference's module surface). Loading
fails loudly when libllgpu.so is missing: there is no CPU path behind it.
"""
from __future__ import annotations

import ctypes
import os
import re

from . import LIB_PATH, PKG_DIR

HEADER = os.path.join(os.path.dirname(PKG_DIR), "include", "llgpu.h")

ENGINES = {"fp64": 0, "ntt": 1}
STATUS = {0: "LLG_OK", 1: "LLG_E_CUDA", 2: "LLG_E_NODEV", 3: "LLG_E_ARG", 4: "LLG_E_UNSUPPORTED",
          5: "LLG_E_ROUNDOFF", 6: "LLG_E_TIMEOUT", 7: "LLG_E_NOMEM"}


class LlgResult(ctypes.Structure):
    _fields_ = [("p", ctypes.c_uint64), ("iters", ctypes.c_uint64), ("res64", ctypes.c_uint64),
                ("max_err", ctypes.c_double), ("seconds", ctypes.c_double), ("n", ctypes.c_uint32),
                ("escalations", ctypes.c_uint32), ("is_zero", ctypes.c_int32), ("status", ctypes.c_int32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class LlgError(RuntimeError):
    def __init__(self, code, detail=""):
        self.code = code
        super().__init__(f"{STATUS.get(code, code)}: {detail}")


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run mersenneprime_python_cpp_gmp_benchmark_b200.build()")
        L = ctypes.CDLL(LIB_PATH)
        u64, u32, i32, dbl, sz = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int32, ctypes.c_double, ctypes.c_size_t
        P = ctypes.POINTER
        L.llg_status_string.argtypes = [ctypes.c_int]
        L.llg_status_string.restype = ctypes.c_char_p
        L.llg_last_error.argtypes = []
        L.llg_last_error.restype = ctypes.c_char_p
        L.llg_device_info.argtypes = [ctypes.c_char_p, sz, P(ctypes.c_int), P(u64)]
        L.llg_fft_length.argtypes = [u64, dbl]
        L.llg_fft_length.restype = u32
        L.llg_set_max_bpw.argtypes = [dbl]
        L.llg_set_roundoff_limit.argtypes = [dbl]
        L.llg_set_length_choice.argtypes = [u32, u32]
        L.llg_get_length_choice.argtypes = [u32]
        L.llg_get_length_choice.restype = u32
        L.llg_get_roundoff_limit.argtypes = []
        L.llg_get_roundoff_limit.restype = dbl
        L.llg_get_max_bpw.restype = dbl
        L.llg_ntt_length.argtypes = [u64]
        L.llg_ntt_length.restype = u32
        L.llg_max_exponent.argtypes = [ctypes.c_int]
        L.llg_max_exponent.restype = u64
        L.llg_run.argtypes = [u64, u64, ctypes.c_int, u32, P(LlgResult), P(u64), sz]
        L.llg_run_batch.argtypes = [P(u64), sz, u64, ctypes.c_int, P(LlgResult), P(u64), sz]
        L.llg_residue_from_digits.argtypes = [u64, u32, P(ctypes.c_int64), P(u64), sz, P(u64), P(i32)]
        L.llg_batch_create.argtypes = [P(u64), sz, u64, ctypes.c_int, ctypes.c_int, P(ctypes.c_void_p)]
        L.llg_batch_launch.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.llg_batch_results.argtypes = [ctypes.c_void_p, P(LlgResult), P(u64), sz]
        L.llg_batch_errlog.argtypes = [ctypes.c_void_p, P(ctypes.c_float), sz, P(sz)]
        L.llg_measure_peak.argtypes = [ctypes.c_int, P(dbl)]
        L.llg_h2d_bytes.argtypes = []
        L.llg_h2d_bytes.restype = u64
        L.llg_release_cached.argtypes = []
        L.llg_release_cached.restype = None
        L.llg_batch_device_ms.argtypes = [ctypes.c_void_p, P(ctypes.c_float)]
        L.llg_batch_destroy.argtypes = [ctypes.c_void_p]
        L.llg_run_noalloc.argtypes = [u64, u64, u32, ctypes.c_void_p, P(dbl), ctypes.c_void_p]
        L.llg_test_create.argtypes = [u64, u32, ctypes.c_int, P(ctypes.c_void_p)]
        L.llg_test_start.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.llg_test_iterate.argtypes = [ctypes.c_void_p, u64, ctypes.c_void_p]
        L.llg_test_read.argtypes = [ctypes.c_void_p, ctypes.c_void_p, P(LlgResult), P(u64), sz]
        L.llg_test_errlog.argtypes = [ctypes.c_void_p, P(ctypes.c_float), sz, P(sz)]
        L.llg_set_large_split.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.llg_get_large_split.argtypes = [ctypes.c_int, P(ctypes.c_int)]
        L.llg_residue_from_digits_device.argtypes = [u64, u32, ctypes.c_void_p, ctypes.c_void_p, P(u64),
                                                     P(ctypes.c_int32), ctypes.c_void_p]
        L.llg_test_time_passes.argtypes = [ctypes.c_void_p, u64, ctypes.c_void_p, P(ctypes.c_double),
                                           P(ctypes.c_double)]
        L.llg_test_destroy.argtypes = [ctypes.c_void_p]
        L.llg_test_load.argtypes = [ctypes.c_void_p, P(u64), sz, u64, ctypes.c_void_p]
        L.llg_test_diag_withhold_wrap.argtypes = [ctypes.c_void_p, u64, ctypes.c_void_p]
        L.llg_test_destroy.restype = None
        L.llg_batch_destroy.restype = None
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise LlgError(rc, (lib().llg_last_error() or b"").decode())


def header_functions():
    """Names of the functions include/llgpu.h declares."""
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(llg_[a-z_0-9]+)\s*\(", src, re.M)))


def nwords(p):
    return max(1, (p + 63) // 64)


def device_info():
    name = ctypes.create_string_buffer(256)
    sms, mem = ctypes.c_int(), ctypes.c_uint64()
    _check(lib().llg_device_info(name, 256, ctypes.byref(sms), ctypes.byref(mem)))
    return name.value.decode(), sms.value, mem.value


def measure_peak(which="fp64"):
    """Measured ops/s: 'fp64' FMA flops/s or 'int32' multiply-adds/s."""
    v = ctypes.c_double()
    _check(lib().llg_measure_peak(0 if which == "fp64" else 1, ctypes.byref(v)))
    return v.value


def h2d_bytes():
    """Bytes the library has copied from host to device since it was loaded (all threads)."""
    return int(lib().llg_h2d_bytes())


def release_cached():
    """Frees the two-pass test llg_run keeps for a repeated call on the same exponent."""
    lib().llg_release_cached()


def fft_length(p, max_bpw=0.0):
    return int(lib().llg_fft_length(p, max_bpw))


def ntt_length(p):
    return int(lib().llg_ntt_length(p))


def set_roundoff_limit(limit):
    """llg_set_roundoff_limit: the FP64 round-off bound above which a test is redone longer."""
    _check(lib().llg_set_roundoff_limit(limit))


def get_roundoff_limit():
    return lib().llg_get_roundoff_limit()


def set_length_choice(n_rule, n_use):
    """llg_set_length_choice: where the bits-per-digit rule gives the whole-test length n_rule, use
    n_use (0: the rule's own)."""
    _check(lib().llg_set_length_choice(n_rule, n_use))


def get_length_choice(n_rule):
    return lib().llg_get_length_choice(n_rule)


def _usable_lengths(p, lo, count):
    """The FP64 lengths >= lo usable for p, ascending (at most count): llg_fft_length at a falling
    bits-per-digit bound walks up the ladder of lengths."""
    out, bpw = [], p / lo
    while len(out) < count and bpw > 2.0:
        n = fft_length(p, bpw)
        if n and n >= lo and n not in out:
            out.append(n)
        bpw *= 0.97
    return sorted(out)


def autotune_range(hi=100001, iters=1000, tests=444, candidates=3, save=True, path=None):
    """Times, for every whole-test length N the bits-per-digit rule picks for the primes p <= hi,
    a batch of that bucket's largest exponents (`tests` of them, one block each, `iters` squarings)
    at N and at the next usable whole-test lengths (up to `candidates` in all), keeps the fastest
    in force (llg_set_length_choice) and, with `save`, records it in the tune file.
    Returns {N: (chosen, {candidate: device ms})}."""
    name = device_info()[0]
    buckets, old = {}, {}
    for p in _primes(3, hi):
        n = fft_length(p)
        if n and n <= 12288:
            buckets.setdefault(n, []).append(p)
    for n in buckets:
        old[n] = get_length_choice(n)
        set_length_choice(n, 0)
    out = {}
    try:
        for n, bp in sorted(buckets.items()):
            sample = sorted(bp)[-tests:]
            # whole-test lengths only (a two-pass length would run the bucket one exponent at a time)
            cands = [c for c in _usable_lengths(sample[0], n, candidates) if c <= 12288]
            times = {}
            for c in cands:
                set_length_choice(n, c)
                b = Batch(sample, iters)
                try:
                    b.launch()
                    b.device_ms()
                    b.launch()
                    times[c] = b.device_ms()
                finally:
                    b.close()
            set_length_choice(n, 0)
            out[n] = (min(times, key=times.get) if times else n, times)
        for n, (best, _) in out.items():
            set_length_choice(n, best)
    except Exception:
        for n, c in old.items():
            set_length_choice(n, c)
        raise
    if save:
        path = path or tune_cache_path()
        keep = []
        if os.path.exists(path):
            with open(path) as f:
                for line in f:
                    fl = line.rstrip("\n").split("\t")
                    if len(fl) >= 3 and fl[0] == "length" and fl[1] == name and int(fl[2]) in out:
                        continue
                    keep.append(line.rstrip("\n"))
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            for line in keep:
                f.write(line + "\n")
            for n, (best, _) in sorted(out.items()):
                f.write(f"length\t{name}\t{n}\t{best}\n")
        os.replace(tmp, path)
    return out


def set_large_split(log_n, log_c, rows=0):
    """Shape of the two-pass FP64 engine at N = 2^log_n: rows of 2^log_c complex values, `rows` rows
    per row-pass block (0: the default for log_c); log_c = -1 restores the built-in shape."""
    _check(lib().llg_set_large_split(log_n, log_c, rows))


def get_large_split(log_n):
    """(log2 row length, rows per block) in force at N = 2^log_n."""
    rows = ctypes.c_int()
    lc = lib().llg_get_large_split(log_n, ctypes.byref(rows))
    return lc, rows.value


def large_splits(log_n):
    """The (log2 row length, rows per block) shapes the two-pass FP64 kernels implement at 2^log_n."""
    old = get_large_split(log_n)
    ok = [(c, g) for c in range(6, 12) for g in (4, 2, 8) if lib().llg_set_large_split(log_n, c, g) == 0]
    set_large_split(log_n, *old)
    return ok


def tune_cache_path():
    """Where the autotuner's choices live ($LLG_TUNE_CACHE, else ~/.cache/llgpu/tune.txt); the
    library reads the file once per process, on its first device call."""
    return os.environ.get("LLG_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "llgpu",
                                                             "tune.txt")


def autotune(log_ns=range(14, 24), iters=64, warmup=16, save=True, path=None):
    """Times every shape (row x column split, rows per row-pass block) of the two-pass FP64 engine
    at each length N = 2^log_n on this GPU (one exponent at ~16.5 bits/digit, `iters` squarings
    pass by pass after `warmup`), keeps the fastest in force (llg_set_large_split) and, with
    `save`, records it in the tune file for later processes.
    Returns {log_n: ((log_c, rows), {(log_c, rows): us per squaring})}."""
    name = device_info()[0]
    out = {}
    for ln in log_ns:
        n = 1 << ln
        p = int(16.5 * n) | 1
        times = {}
        for c in large_splits(ln):
            set_large_split(ln, *c)
            t = Test(p, n)
            try:
                t.start()
                t.iterate(warmup)
                r, k = t.time_passes(iters)
                times[c] = r + k
            finally:
                t.close()
        best = min(times, key=times.get)
        set_large_split(ln, *best)
        out[ln] = (best, times)
    if save:
        path = path or tune_cache_path()
        keep = []
        if os.path.exists(path):
            with open(path) as f:
                for line in f:
                    fl = line.rstrip("\n").split("\t")
                    if len(fl) >= 4 and fl[0] == "large_split" and fl[1] == name and int(fl[2]) in out:
                        continue
                    keep.append(line.rstrip("\n"))
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            for line in keep:
                f.write(line + "\n")
            for ln, (best, _) in sorted(out.items()):
                f.write(f"large_split\t{name}\t{ln}\t{best[0]}\t{best[1]}\n")
        os.replace(tmp, path)
    return out


def run(p, iters=0, engine="fp64", n=0, want_words=False):
    """One test (or its first `iters` squarings) -> dict of llg_result fields (+ 'words')."""
    r = LlgResult()
    words = (ctypes.c_uint64 * nwords(p))() if want_words else None
    _check(lib().llg_run(p, iters, ENGINES[engine], n, ctypes.byref(r), words, nwords(p) if want_words else 0))
    d = r.as_dict()
    if want_words:
        d["words"] = list(words)
    return d


def run_batch(ps, iters=0, engine="fp64", want_words=False):
    ps = list(ps)
    arr = (ctypes.c_uint64 * len(ps))(*ps)
    out = (LlgResult * len(ps))()
    total = sum(nwords(p) for p in ps)
    words = (ctypes.c_uint64 * total)() if want_words else None
    _check(lib().llg_run_batch(arr, len(ps), iters, ENGINES[engine], out, words, total if want_words else 0))
    res = [o.as_dict() for o in out]
    if want_words:
        off = 0
        for d, p in zip(res, ps):
            d["words"] = list(words[off:off + nwords(p)])
            off += nwords(p)
    return res


class Batch:
    """A device-resident batch (llg_batch_*): create once, launch on a stream, read results."""

    KEEP_WORDS, ERRLOG = 1, 2

    def __init__(self, ps, iters=0, engine="fp64", flags=0):
        self.ps = list(ps)
        arr = (ctypes.c_uint64 * len(self.ps))(*self.ps)
        self.h = ctypes.c_void_p()
        self.flags = flags
        _check(lib().llg_batch_create(arr, len(self.ps), iters, ENGINES[engine], flags, ctypes.byref(self.h)))

    def launch(self, stream=0):
        """Enqueue on a CUDA stream handle (int, e.g. torch.cuda.Stream.cuda_stream; 0 = internal)."""
        _check(lib().llg_batch_launch(self.h, ctypes.c_void_p(stream or None)))

    def results(self, want_words=False):
        out = (LlgResult * len(self.ps))()
        total = sum(nwords(p) for p in self.ps)
        words = (ctypes.c_uint64 * total)() if want_words else None
        _check(lib().llg_batch_results(self.h, out, words, total if want_words else 0))
        res = [o.as_dict() for o in out]
        if want_words:
            off = 0
            for d, p in zip(res, self.ps):
                d["words"] = list(words[off:off + nwords(p)])
                off += nwords(p)
        return res

    def device_ms(self):
        ms = ctypes.c_float()
        _check(lib().llg_batch_device_ms(self.h, ctypes.byref(ms)))
        return ms.value

    def errlog(self):
        n = self.ps and max(self.ps) or 0
        buf = (ctypes.c_float * n)()
        ln = ctypes.c_size_t()
        _check(lib().llg_batch_errlog(self.h, buf, n, ctypes.byref(ln)))
        return list(buf[:ln.value])

    def close(self):
        if self.h:
            lib().llg_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Test:
    """One exponent on the two-pass engine (llg_test_*): start, iterate on a stream, read."""

    def __init__(self, p, n=0, engine="fp64"):
        self.p = p
        self.h = ctypes.c_void_p()
        _check(lib().llg_test_create(p, n, ENGINES[engine], ctypes.byref(self.h)))

    def start(self, stream=0):
        _check(lib().llg_test_start(self.h, ctypes.c_void_p(stream or None)))

    def iterate(self, iters, stream=0):
        _check(lib().llg_test_iterate(self.h, iters, ctypes.c_void_p(stream or None)))

    def read(self, stream=0, want_words=False):
        r = LlgResult()
        nw = nwords(self.p)
        words = (ctypes.c_uint64 * nw)() if want_words else None
        _check(lib().llg_test_read(self.h, ctypes.c_void_p(stream or None), ctypes.byref(r), words,
                                   nw if want_words else 0))
        d = r.as_dict()
        if want_words:
            d["words"] = list(words)
        return d

    def load(self, words, iters_done, stream=0):
        """llg_test_load: the state becomes the residue `words` (ceil(p/64) limbs) after
        `iters_done` squarings, and the next squaring starts."""
        nw = nwords(self.p)
        arr = (ctypes.c_uint64 * nw)(*words[:nw])
        _check(lib().llg_test_load(self.h, arr, nw, iters_done, ctypes.c_void_p(stream or None)))

    def diag_withhold_wrap(self, spin_limit, stream=0):
        """llg_test_diag_withhold_wrap: one row pass whose waits must run out (raises LlgError)."""
        _check(lib().llg_test_diag_withhold_wrap(self.h, spin_limit, ctypes.c_void_p(stream or None)))

    def time_passes(self, iters, stream=0):
        """`iters` squarings one pass at a time: (mean row-pass us, mean column-pass us)."""
        r, c = ctypes.c_double(), ctypes.c_double()
        _check(lib().llg_test_time_passes(self.h, iters, ctypes.c_void_p(stream or None), ctypes.byref(r),
                                          ctypes.byref(c)))
        return r.value, c.value

    def errlog(self, n):
        buf = (ctypes.c_float * n)()
        ln = ctypes.c_size_t()
        _check(lib().llg_test_errlog(self.h, buf, n, ctypes.byref(ln)))
        return list(buf[:ln.value])

    def close(self):
        if self.h:
            lib().llg_test_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_noalloc(p, iters, n, digits_dev_ptr, stream=0):
    """llg_run_noalloc: squarings without device allocation; digits land in the caller's device
    buffer (n int32). Returns the worst round-off."""
    err = ctypes.c_double()
    _check(lib().llg_run_noalloc(p, iters, n, ctypes.c_void_p(digits_dev_ptr), ctypes.byref(err),
                                 ctypes.c_void_p(stream or None)))
    return err.value


def residue_from_digits_device(p, n, digits_dev_ptr, want_words=False, stream=0):
    """llg_residue_from_digits_device: the residue of n int32 digits in device memory, rebuilt on
    the GPU. Returns (is_zero, res64, words or None); words go through a temporary device buffer."""
    r64, z = ctypes.c_uint64(), ctypes.c_int32()
    if not want_words:
        _check(lib().llg_residue_from_digits_device(p, n, ctypes.c_void_p(digits_dev_ptr), None, ctypes.byref(r64),
                                                    ctypes.byref(z), ctypes.c_void_p(stream or None)))
        return bool(z.value), r64.value, None
    import torch
    dw = torch.empty(nwords(p), dtype=torch.int64, device="cuda")
    _check(lib().llg_residue_from_digits_device(p, n, ctypes.c_void_p(digits_dev_ptr), ctypes.c_void_p(dw.data_ptr()),
                                                ctypes.byref(r64), ctypes.byref(z), ctypes.c_void_p(stream or None)))
    words = [w & 0xFFFFFFFFFFFFFFFF for w in dw.cpu().tolist()]
    return bool(z.value), r64.value, words


def residue_from_digits(p, n, digits):
    d = (ctypes.c_int64 * n)(*[int(x) for x in digits])
    words = (ctypes.c_uint64 * nwords(p))()
    r64, z = ctypes.c_uint64(), ctypes.c_int32()
    _check(lib().llg_residue_from_digits(p, n, d, words, nwords(p), ctypes.byref(r64), ctypes.byref(z)))
    return bool(z.value), r64.value, list(words)


def _primes(lo, hi):
    comp = bytearray(hi + 1)
    for i in range(2, int(hi ** 0.5) + 1):
        if not comp[i]:
            comp[i * i::i] = b"\x01" * len(range(i * i, hi + 1, i))
    return [i for i in range(max(lo, 2), hi + 1) if not comp[i]]


def _main(argv=None):
    """`python -m mersenneprime_python_cpp_gmp_benchmark_b200.llgpu square|batch ...`: one
    exponent's squarings on a two-pass engine, or a batch of whole tests; prints one JSON line
    (res64, worst round-off, wall seconds). Small, self-contained runs for timing and profiling."""
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser(prog="llgpu")
    sub = ap.add_subparsers(dest="cmd", required=True)
    a = sub.add_parser("square", help="k squarings of one exponent from s_0 = 4 (llg_test_*)")
    a.add_argument("--p", type=int, required=True)
    a.add_argument("--iters", type=int, default=8)
    a.add_argument("--n", type=int, default=0)
    a.add_argument("--engine", choices=tuple(ENGINES), default="fp64")
    a.add_argument("--shape", default="", help="two-pass FP64 shape 'log2 row length,rows per block'")
    b = sub.add_parser("batch", help="whole Lucas-Lehmer tests of every prime in [lo, hi]")
    b.add_argument("--lo", type=int, required=True)
    b.add_argument("--hi", type=int, required=True)
    b.add_argument("--iters", type=int, default=0, help="squarings per test (0 = all p-2)")
    b.add_argument("--engine", choices=tuple(ENGINES), default="fp64")
    args = ap.parse_args(argv)
    t0 = time.perf_counter()
    if args.cmd == "square":
        if args.shape:
            c, g = (int(x) for x in args.shape.split(","))
            n = args.n or fft_length(args.p)
            set_large_split(n.bit_length() - 1, c, g)
        t = Test(args.p, args.n, args.engine)
        t.start()
        if args.iters > 1:
            t.iterate(args.iters - 1)
        r = t.read()
        t.close()
        out = {"p": args.p, "n": r["n"], "iters": r["iters"], "res64": f"{r['res64']:016x}",
               "max_err": r["max_err"], "engine": args.engine}
    else:
        ps = _primes(args.lo, args.hi)
        rs = run_batch(ps, args.iters, args.engine)
        out = {"tests": len(ps), "hits": [r["p"] for r in rs if r["is_zero"]],
               "failed": [r["p"] for r in rs if r["status"]], "engine": args.engine,
               "lengths": sorted({r["n"] for r in rs})}
    out["seconds"] = round(time.perf_counter() - t0, 3)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(_main())
