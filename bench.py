#!/usr/bin/env python3
"""Benchmark of the B200 Lucas-Lehmer engine; prints ONE JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload big|range] [--impl b200|reference]

Workloads (synthetic inputs: the exponents themselves, s_0 = 4; no dataset exists for this path):
  big     (default) p = 136,279,841 on the two-pass FP64 IBDWT engine at N = 2^23; one step = 1000
          squarings. metric: us per Lucas-Lehmer iteration (lower is better). value: CUDA events on
          the launch stream, the 64 MiB state resident on the device, L2 flushed between steps.
          e2e: lucaslehmer.fft_res64_after(p, 2000) as a cold call -- tables built and uploaded,
          buffers allocated, s_0 set on the device, graphs captured, squarings, exact residue
          rebuilt on the device, res64 back -- per squaring; beside it the same call repeated on
          the two-pass test the library keeps. Host-to-device bytes are the library's own count.
          The line also carries the other half of the metric as "range" (the range workload below,
          one timed step; leave it out with --no-range).
  range   every prime p <= 100,001 (9,592 Lucas-Lehmer tests, 28 Mersenne hits), batched whole-test
          kernels bucketed by transform length. One step = every test run to completion.
          metric: tests/s. e2e: lucaslehmer_cuda.lucas_lehmer_batch() on the host list.
          batched_vs_plain: every prime p <= 10,001 one exponent per launch against one batched
          launch, on the same GPU (device time, residues compared). reference_gpu: the reference's
          own cuda/ll_ntt.cu (compiled unchanged for sm_100a) on a sample of the range, same GPU.
  single  p = 1,257,787 (a Mersenne exponent) at N = 65536, the whole test on the FP64 and NTT
          engines: us per squaring, res64 every 10^4 squarings against the reference GMP trace,
          final residue zero, the round-off maximum and per-squaring log.
  sweep   8 seeded primes in [20M, 25M]: FP64 asked at N = 2^20 (escalating on round-off > 0.4)
          against the NTT at its exact length; length used, escalations, round-off, us per squaring.
--impl reference: the reference's own CPU engines (its lucaslehmer.cpp compiled unchanged into
oracle/_ref/) on the host cores for the same metric: bench_square at p = 136,279,841 (big; with
the range sample beside it) or a stratified sample of the range (range), GMP engine as the value
and FFT engine beside it. FFTW3 is absent, so the reference FFT engine runs over the oracle's
radix-2 FFT; its published FFTW figure for the range is quoted with it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "mersenneprime_python_cpp_gmp_benchmark_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

RANGE_HI = 100001
METRIC_RANGE = "tests/s for all p<=100001 (residues exact)"
BIG_P = 136279841
METRIC_BIG = "us/LL-iteration at p=136,279,841"
STEP_ITERS = 1000  # squarings per timed step of the p=136,279,841 workload
PASS_ITERS = 100   # squarings timed pass by pass for the dominant kernel's roofline
# DRAM bytes (read + write) of one launch at p=136,279,841, N=2^23, from an ncu capture of
# `python -m mersenneprime_python_cpp_gmp_benchmark_b200.llgpu square --p 136279841 --n 8388608
# --iters 6 --shape 10,8` (NTT: `... --iters 6 --engine ntt`). ncu captures run cold (caches
# flushed), so these are upper bounds on a warm launch, where part of the 64 MiB state is still in L2.
NCU_TRAFFIC = {"fp64": {"row": 89817600, "column": 76730880},
               "ntt": {"row": 115433728, "column": 94066176}}


def sieve(lo, hi):
    comp = bytearray(hi + 1)
    i = 2
    while i * i <= hi:
        if not comp[i]:
            comp[i * i::i] = b"\x01" * len(range(i * i, hi + 1, i))
        i += 1
    return [i for i in range(max(lo, 2), hi + 1) if not comp[i]]


# ---- clocks sampled during the timed region ------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---- distributed plumbing ------------------------------------------------------------------

def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=600))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    from mersenneprime_python_cpp_gmp_benchmark_b200 import replicas
    return replicas.reduce_max(x) if world > 1 else x


def sum_over_ranks(x, world):
    from mersenneprime_python_cpp_gmp_benchmark_b200 import replicas
    return replicas.reduce_sum(x) if world > 1 else x


class L2Flush:
    """Writes a buffer larger than the 126 MB L2 between timed steps."""

    def __init__(self):
        import torch
        self.buf = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def __call__(self):
        import torch
        self.buf.fill_(1.0)
        torch.cuda.synchronize()


# ---- the range workload ------------------------------------------------------------------

def range_flops(results):
    """Algorithmic FP64 flops of the tests: 5 N log2 N per squaring (forward + inverse real FFT)."""
    import math
    tot = 0.0
    for r in results:
        n = r["n"]
        if n >= 32:
            tot += r["iters"] * 5.0 * n * math.log2(n)
    return tot


def plain_vs_batched(llgpu, hi=10001):
    """Every prime p <= hi (1229 tests for 10001) as one exponent per launch, then as one batched
    launch, on the same GPU: device time of the launches, residues compared."""
    ps = sieve(2, hi)
    batch = llgpu.Batch(ps)
    batch.launch()
    batch.device_ms()
    batch.launch()
    t_batch = batch.device_ms() * 1e-3
    res = {r["p"]: r["res64"] for r in batch.results()}
    batch.close()
    t_plain = 0.0
    for p in ps:
        one = llgpu.Batch([p])
        one.launch()
        t_plain += one.device_ms() * 1e-3
        assert one.results()[0]["res64"] == res[p], f"p={p}: per-exponent and batched residues differ"
        one.close()
    return {"tests": f"every prime p <= {hi} ({len(ps)} tests), one exponent per launch vs one batched launch",
            "plain_tests_per_s": round(len(ps) / t_plain, 2), "batched_tests_per_s": round(len(ps) / t_batch, 2),
            "batched_speedup": round(t_plain / t_batch, 2), "timing": "device time of the launches (CUDA events)"}


def bench_range(args, rank, world):
    import torch
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    ps_all = sieve(2, RANGE_HI)
    # the range autotuner picks, per whole-test length of the bits-per-digit rule, the fastest of
    # that length and the next usable ones on this GPU (power of two against {3,5} x 2^k);
    # --range-lengths rule keeps the rule's lengths (a profiler's timings would mislead it)
    if getattr(args, "range_lengths", "tuned") == "rule":
        for n in {llgpu.fft_length(p) for p in ps_all if p > 2}:
            if 0 < n <= 12288:
                llgpu.set_length_choice(n, 0)
        tuned = {}
    else:
        tuned = llgpu.autotune_range(RANGE_HI, save=False)
    from mersenneprime_python_cpp_gmp_benchmark_b200 import replicas
    mine = replicas.shard(ps_all, rank, world)  # independent tests, balanced by squaring cost
    batch = llgpu.Batch(mine)
    flush = L2Flush()
    for _ in range(args.warmup):
        batch.launch()
        batch.device_ms()
    res = batch.results()
    known = {int(x) for x in open(os.path.join(ROOT, "tests", "golden", "known_mp_list.txt")).read().split()}
    hits = sorted(r["p"] for r in res if r["is_zero"])
    assert all(r["status"] == 0 for r in res), "a test failed"
    assert set(hits) == {p for p in known if p in set(mine)}, "hit set differs from known_mp_list.txt"
    barrier(world)
    torch.cuda.synchronize()
    times = []
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for _ in range(args.steps):
            flush()
            batch.launch()
            times.append(batch.device_ms() * 1e-3)
    torch.cuda.synchronize()
    barrier(world)
    t_rank = sum(times)
    t_max = max_over_ranks(t_rank, world)
    tests = sum_over_ranks(len(mine) * args.steps, world)
    value = tests / t_max
    # e2e through the reference-facing call (host lists in, results out)
    import lucaslehmer_cuda as lc
    lc.lucas_lehmer_batch(mine[:64])
    h0 = llgpu.h2d_bytes()
    t0 = time.perf_counter()
    out = lc.lucas_lehmer_batch(mine)
    t_e2e = time.perf_counter() - t0
    h2d = llgpu.h2d_bytes() - h0
    assert sorted(p for p, r, s, res64 in out if r) == hits
    t_e2e = max_over_ranks(t_e2e, world)
    e2e = sum_over_ranks(len(mine), world) / t_e2e
    # up: measured by the library's count (the job lists and word offsets); back: each test's
    # result record, res64 and zero flag (the residue is rebuilt on the device)
    d2h = (32 + 8 + 4) * len(mine)
    flops = range_flops(res)
    achieved = flops / (t_rank / args.steps) / 1e12
    peak = llgpu.measure_peak("fp64") / 1e12
    line = {
        "metric": METRIC_RANGE, "value": round(value, 2), "unit": "tests/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * t_max / args.steps, 3),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: every prime exponent p <= 100001 from the sieve, s_0 = 4",
        "config": {"workload": "range p<=100001 (9592 LL tests, batched whole-test kernels, FP64 IBDWT, "
                               "N = {1,3,5} x 2^k from 32 to 6144 at <=18 bits/digit)",
                   "lengths": {str(n): c for n, c in sorted(__import__("collections").Counter(r["n"] for r in res).items())},
                   "tests": len(ps_all), "l2": "flushed (512 MiB write) between steps",
                   "autotuned_lengths": {str(n): {"use": best, "candidates_ms": {str(c): round(v, 2) for c, v in t.items()}}
                                         for n, (best, t) in tuned.items()},
                   "parallelism": f"independent tests split over {world} GPU(s) by squaring cost (replicas)"},
        "e2e": {"value": round(e2e, 2), "unit": "tests/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "fp64", "achieved": round(achieved, 3), "peak": round(peak, 3), "unit": "TFLOP/s",
                     "frac": round(achieved / peak, 4),
                     "peak_source": "measured FP64 FMA probe (llg_measure_peak)", "traffic": None,
                     "work": "5 N log2 N flops per squaring x (p-2) squarings, summed over the range"},
        "clocks": clk.summary(),
        "hits": len(hits),
        "gpu_launches": args.steps * len({r["n"] for r in res}),
    }
    if rank == 0:
        line["batched_vs_plain"] = plain_vs_batched(llgpu)
        if not getattr(args, "no_reference_gpu", False):
            line["reference_gpu"] = reference_gpu_range()
    return line


def bench_big(args, rank, world):
    """p = 136,279,841 on a two-pass engine at N = 2^23; one step = 1000 squarings."""
    import torch
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    n = 1 << 23
    tuned = None
    if args.engine == "fp64" and args.split:
        # a fixed split (a profiler's timings would mislead the autotuner)
        c, g = (int(x) for x in args.split.split(","))
        llgpu.set_large_split(23, c, g)
        tuned = {"row_length": f"2^{c} complex", "column_length": f"2^{22 - c} complex", "rows_per_block": g,
                 "candidates_us": None, "fixed": True}
    elif args.engine == "fp64":
        # the autotuner picks the row x column split of the two-pass engine on this GPU
        best, cand = llgpu.autotune([23], save=False)[23]
        tuned = {"row_length": f"2^{best[0]} complex", "column_length": f"2^{22 - best[0]} complex",
                 "rows_per_block": best[1],
                 "candidates_us": {f"2^{c}x2^{22 - c}/{g}": round(v, 2) for (c, g), v in cand.items()}}
    stream = torch.cuda.Stream()
    handle = stream.cuda_stream
    t = llgpu.Test(BIG_P, n, args.engine)
    t.start(handle)
    flush = L2Flush()
    for _ in range(args.warmup):
        t.iterate(STEP_ITERS, handle)
    torch.cuda.synchronize()
    barrier(world)
    times = []
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for _ in range(args.steps):
            flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t.iterate(STEP_ITERS, handle)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1) * 1e-3)
    torch.cuda.synchronize()
    barrier(world)
    # the dominant kernel's own time: PASS_ITERS squarings launched one pass at a time, CUDA events
    # between the launches on the launch stream
    row_us, col_us = t.time_passes(PASS_ITERS, handle)
    done = 1 + STEP_ITERS * (args.warmup + args.steps) + PASS_ITERS
    r = t.read(handle)
    assert r["iters"] == done and r["status"] == 0, r
    t.close()
    t_rank = sum(times)
    t_max = max_over_ranks(t_rank, world)
    # whole job: `world` independent replicas each did STEP_ITERS * steps squarings in <= t_max
    us_iter = 1e6 * t_max / (STEP_ITERS * args.steps * world)
    # correctness of the timed engine: res64 after 1000 squarings vs the reference GMP engine
    gold = {(d["p"], d["k"]): int(d["res64"], 16)
            for d in json.load(open(os.path.join(ROOT, "tests", "golden", "appendix.json")))["after"]}
    chk = llgpu.run(BIG_P, iters=1000, n=n, engine=args.engine)
    assert chk["res64"] == gold[(BIG_P, 1000)], "res64 after 1000 squarings differs from the reference"
    # e2e: the reference-facing call, host in / host out, for a 2000-squaring interim residue
    import lucaslehmer as ll
    k_e2e = 2000

    def e2e_call():
        h0 = llgpu.h2d_bytes()
        t0 = time.perf_counter()
        if args.engine == "fp64":
            ll.fft_res64_after(BIG_P, k_e2e)
        else:
            ll.gmp_res64_after(BIG_P, k_e2e)  # the exact call; the NTT engine serves it
        return max_over_ranks(time.perf_counter() - t0, world), llgpu.h2d_bytes() - h0

    # a cold call (the two-pass test kept by the check run above released first: tables built and
    # uploaded, buffers allocated, graphs captured inside the timed call), then the same call again
    llgpu.release_cached()
    t_e2e, h2d_e2e = e2e_call()
    reps = [e2e_call() for _ in range(3)]
    t_rep, h2d_rep = statistics.median(x[0] for x in reps), max(x[1] for x in reps)
    bytes_iter = 32.0 * n   # two read+write sweeps of the 8N-byte state
    bytes_pass = 16.0 * n   # one pass reads and writes the 8N-byte state once
    flops_iter = 5.0 * n * 23
    dom, dom_us = ("row", row_us) if row_us >= col_us else ("column", col_us)
    traffic = NCU_TRAFFIC[args.engine][dom]
    peaks_file = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_file):
        hbm_peak = json.load(open(peaks_file))["hbm_gbs"]
        peak_source = "measured (MEASURED_PEAKS.json hbm_gbs, burst copy)"
    else:
        hbm_peak = 6650.0
        peak_source = "fallback: 6.65 TB/s, an earlier copy measurement on this GPU pool"
    achieved = bytes_iter / (us_iter * world * 1e-6) / 1e9  # per GPU
    fp64_peak = llgpu.measure_peak("fp64") / 1e12
    line = {
        "metric": METRIC_BIG, "value": round(us_iter, 3), "unit": "us/iteration", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * t_max / args.steps, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.engine == "fp64" else "u64 (GF(2^64-2^32+1))",
        "data": "synthetic: the LL sequence of p=136,279,841 from s_0=4 (no external data)",
        "config": {"workload": ("p=136,279,841 FP64 IBDWT, N=2^23 (16.25 bits/digit), two-pass "
                                "(rows x columns of 2^22 complex, split autotuned), 1000 squarings per step")
                   if args.engine == "fp64" else
                   ("p=136,279,841 Goldilocks NTT IBDWT, N=2^23 (16.25 bits/digit), two-pass "
                    "(row 1024 x column 8192), 1000 squarings per step"),
                   "engine": args.engine, "autotuned_split": tuned,
                   "l2": "flushed (512 MiB write) between steps; the 64 MiB state stays on device",
                   "parallelism": f"one independent test per GPU ({world} replica(s))"},
        "e2e": {"value": round(1e6 * t_e2e / k_e2e, 3), "unit": "us/iteration", "iters": k_e2e,
                "call": ("lucaslehmer.fft_res64_after" if args.engine == "fp64" else "lucaslehmer.gmp_res64_after")
                        + "(136279841, 2000), cold: tables built and uploaded, buffers allocated, s_0 set on "
                          "the device, graphs captured, squarings, exact residue rebuilt on the device, res64 back",
                # measured by the library's own count (llg_h2d_bytes); back: res64, the rebuild's flags
                # and the control block
                "h2d_bytes_per_step": h2d_e2e, "d2h_bytes_per_step": 128,
                "repeat_call": {"value": round(1e6 * t_rep / k_e2e, 3), "unit": "us/iteration",
                                "h2d_bytes": h2d_rep,
                                "note": "the same call again, median of 3: the two-pass test the previous "
                                        "call kept (tables, buffers, graphs) is reused"}},
        "roofline": {"bound": "hbm", "achieved": round(bytes_pass / (dom_us * 1e-6) / 1e9, 1), "peak": hbm_peak,
                     "unit": "GB/s", "frac": round(bytes_pass / (dom_us * 1e-6) / 1e9 / hbm_peak, 4),
                     "peak_source": peak_source,
                     "traffic": traffic,
                     "kernel": f"{dom} pass ({'large' if args.engine == 'fp64' else 'ntt'}_{'row' if dom == 'row' else 'col'})",
                     "kernel_us": round(dom_us, 2), "row_us": round(row_us, 2), "col_us": round(col_us, 2),
                     "work": "16 N bytes per launch (the 8N-byte state read and written once)",
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch"},
        "roofline_iteration": {"achieved": round(achieved, 1), "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                               "work": "32 N bytes per squaring (two read+write sweeps of the 8N-byte state)"},
        "roofline_fp64": {"achieved": round(flops_iter / (us_iter * world * 1e-6) / 1e12, 3),
                          "peak": round(fp64_peak, 3), "unit": "TFLOP/s",
                          "frac": round(flops_iter / (us_iter * world * 1e-6) / 1e12 / fp64_peak, 4),
                          "work": "5 N log2 N flops per squaring", "peak_source": "measured FP64 FMA probe"},
        "max_roundoff": r["max_err"],
        "clocks": clk.summary(),
        "gpu_launches": 2 * STEP_ITERS * args.steps,
    }
    return line


SINGLE_P, SINGLE_N = 1257787, 65536
SWEEP_N = 1 << 20
METRIC_SINGLE = "us/LL-iteration at p=1,257,787 (N=65536, whole test)"
METRIC_SWEEP = "us/LL-iteration over 8 seeded primes in [20M,25M] (FP64 asked at N=2^20)"


def bench_single(args, rank, world):
    """p = 1,257,787 (a Mersenne exponent) at N = 65536 (19.19 bits/digit), every one of its p - 2
    squarings, on the FP64 and the NTT two-pass engines. One step = the whole test. Per engine: us per
    squaring from CUDA events around the squarings (the res64 reads every 10^4 squarings, checked
    against the reference GMP trace, fall outside the events), the final residue (zero), and for
    FP64 the run's worst round-off plus the per-squaring round-off log of its last 65536 squarings.
    The 512 KiB state is L2-resident by design at this size."""
    import torch
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    tr = json.load(open(os.path.join(ROOT, "tests", "golden", "trace_1257787.json")))
    p, every = tr["p"], tr["every"]
    assert p == SINGLE_P
    stream = torch.cuda.Stream()
    h = stream.cuda_stream
    legs = {}
    barrier(world)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for engine in ("fp64", "ntt"):
            w = llgpu.Test(p, SINGLE_N, engine)  # warm-up: tables, graphs, clocks
            w.start(h)
            w.iterate(args.warmup * 1000, h)
            torch.cuda.synchronize()
            w.close()
            t = llgpu.Test(p, SINGLE_N, engine)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

            def timed(fn):
                e0.record(stream)
                fn()
                e1.record(stream)
                e1.synchronize()
                return e0.elapsed_time(e1) * 1e-3

            elapsed = timed(lambda: t.start(h))
            done, checked, mismatches = 1, 0, 0
            for i, want in enumerate(tr["res64"]):
                k = every * (i + 1)
                elapsed += timed(lambda: t.iterate(k - done, h))
                done = k
                r = t.read(h)
                checked += 1
                mismatches += int(r["res64"] != int(want, 16))
            elapsed += timed(lambda: t.iterate(p - 2 - done, h))
            r = t.read(h)
            assert r["iters"] == p - 2 and r["status"] == 0, r
            assert mismatches == 0 and r["is_zero"] == 1, (engine, mismatches, r["res64"])
            leg = {"us_per_iteration": round(1e6 * elapsed / (p - 2), 3), "seconds": round(elapsed, 3),
                   "iterations": p - 2, "final_residue_zero": True,
                   "res64_checked_every": every, "res64_checks": checked, "res64_mismatches": mismatches}
            if engine == "fp64":
                log = sorted(x for x in t.errlog(65536) if x > 0)
                leg["max_roundoff"] = r["max_err"]
                leg["roundoff_log_last_65536"] = {
                    "max": log[-1], "p99": log[int(0.99 * (len(log) - 1))], "median": log[len(log) // 2]}
            t.close()
            legs[engine] = leg
    lead = legs[args.engine]
    t_max = max_over_ranks(lead["seconds"], world)
    us_iter = 1e6 * t_max / ((p - 2) * world)
    # e2e: the C-ABI call llg_run at the same length for an interim residue, host in / host out
    k_e2e = 100000
    llgpu.run(p, iters=1000, n=SINGLE_N, engine=args.engine)
    llgpu.release_cached()  # a cold call: tables and buffers inside the timed region
    h0 = llgpu.h2d_bytes()
    t0 = time.perf_counter()
    e2e_r = llgpu.run(p, iters=k_e2e, n=SINGLE_N, engine=args.engine)
    t_e2e = max_over_ranks(time.perf_counter() - t0, world)
    h2d_e2e = llgpu.h2d_bytes() - h0
    assert e2e_r["iters"] == k_e2e and e2e_r["n"] == SINGLE_N, e2e_r
    return {
        "metric": METRIC_SINGLE, "value": round(us_iter, 3), "unit": "us/iteration", "n_gpus": world,
        "steps": 1, "warmup": args.warmup, "ms_per_step": round(1e3 * t_max, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.engine == "fp64" else "u64 (GF(2^64-2^32+1))",
        "data": "synthetic: the LL sequence of p=1,257,787 from s_0=4 (no external data)",
        "config": {"workload": "p=1,257,787 whole test (1,257,785 squarings) at N=65536 (19.19 bits/digit), "
                               "two-pass engine, FP64 and Goldilocks NTT; one step = the whole test",
                   "engine": args.engine, "l2": "the 512 KiB state is L2-resident by design",
                   "parallelism": f"one independent test per GPU ({world} replica(s))"},
        "engines": legs,
        "e2e": {"value": round(1e6 * t_e2e / k_e2e, 3), "unit": "us/iteration", "iters": k_e2e,
                "call": f"llg_run(1257787, {k_e2e}, {args.engine}, n=65536) through the C-ABI: tables, s_0 upload, "
                        "squarings, residue rebuilt on the device, result struct back",
                "h2d_bytes_per_step": h2d_e2e, "d2h_bytes_per_step": 128},
        "clocks": clk.summary(),
        "gpu_launches": 2 * (p - 2),  # the reported engine's row and column pass per squaring
    }


def bench_sweep(args, rank, world):
    """The 8 seeded primes of [20,000,000, 25,000,000] (sorted(random.Random(0).sample(primes, 8)),
    as listed in tests/golden/appendix.json). FP64 is asked for N = 2^20 (19.4-23.4 bits/digit) and
    escalates to the next length whenever the round-off passes 0.4; the NTT runs at its exact
    length (2^20 up to p = 22,020,096, else 2^21). Per prime and engine: res64 after 1000
    squarings against the reference GMP engine, then a run of K squarings through llg_run: the
    length used, the escalations, the worst round-off and us per squaring (CUDA events of the
    attempt that finished). value = FP64 us per squaring averaged over the 8 primes."""
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "appendix.json")))
    gold = {(d["p"], d["k"]): int(d["res64"], 16) for d in g["after"]}
    primes = g["sweep_primes"]
    iters = {"fp64": args.sweep_iters, "ntt": args.sweep_ntt_iters}
    rows, walls, h2d = [], {"fp64": 0.0, "ntt": 0.0}, {"fp64": 0, "ntt": 0}
    llgpu.run(primes[0], iters=64 * args.warmup, n=SWEEP_N)  # warm-up
    barrier(world)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for p in primes:
            row = {"p": p, "bits_per_digit_at_2^20": round(p / SWEEP_N, 2)}
            for engine in ("fp64", "ntt"):
                n = SWEEP_N if engine == "fp64" else max(SWEEP_N, llgpu.ntt_length(p))
                chk = llgpu.run(p, iters=1000, n=n, engine=engine)
                match = chk["status"] == 0 and chk["res64"] == gold[(p, 1000)]
                llgpu.release_cached()  # each timed run cold: tables and buffers inside it
                h0 = llgpu.h2d_bytes()
                t0 = time.perf_counter()
                r = llgpu.run(p, iters=iters[engine], n=n, engine=engine)
                walls[engine] += time.perf_counter() - t0
                h2d[engine] += llgpu.h2d_bytes() - h0
                assert r["status"] == 0, (p, engine, r)
                row[engine] = {"n_used": r["n"], "escalations": r["escalations"],
                               "max_roundoff": round(r["max_err"], 5),
                               "us_per_iteration": round(1e6 * r["seconds"] / r["iters"], 3),
                               "res64_after_1000_matches_reference": match}
            rows.append(row)
    us = {e: sum(r[e]["us_per_iteration"] for r in rows) / len(rows) for e in ("fp64", "ntt")}
    esc = {e: sum(r[e]["escalations"] for r in rows) for e in ("fp64", "ntt")}
    lead = args.engine
    return {
        "metric": METRIC_SWEEP, "value": round(us[lead], 3), "unit": "us/iteration", "n_gpus": world,
        "steps": 1, "warmup": args.warmup, "ms_per_step": round(1e3 * walls[lead], 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if lead == "fp64" else "u64 (GF(2^64-2^32+1))",
        "data": "synthetic: the LL sequences of 8 seeded primes from s_0=4 (no external data)",
        "config": {"workload": f"precision sweep: 8 primes in [20M,25M], FP64 asked at N=2^20 (escalating on "
                               f"round-off > 0.4) vs NTT at its exact length; {iters['fp64']} FP64 and "
                               f"{iters['ntt']} NTT squarings timed per prime",
                   "engine": lead, "l2": "state 16-32 MiB per test; one test at a time",
                   "parallelism": "one GPU"},
        "primes": rows,
        "mean_us_per_iteration": {e: round(v, 3) for e, v in us.items()},
        "escalations_total": esc,
        "res64_mismatches": sum(not r[e]["res64_after_1000_matches_reference"] for r in rows for e in ("fp64", "ntt")),
        "e2e": {"value": round(1e6 * walls[lead] / (iters[lead] * len(primes)), 3), "unit": "us/iteration",
                "call": "llg_run(p, K, engine, n) per prime through the C-ABI: tables, s_0 upload, every "
                        "attempt (escalations included), residue rebuilt on the device, result struct back",
                "h2d_bytes_per_step": h2d[lead], "d2h_bytes_per_step": 128 * len(primes)},
        "clocks": clk.summary(),
    }


def cpu_baseline_interim(p, k0, k1, what):
    """Reference GMP engine (oracle/_ref, compiled unchanged) per squaring at p, from
    gmp_res64_after(p, k1) - gmp_res64_after(p, k0): one core."""
    from oracle import oracle
    ref = oracle.reference_module()
    if ref is None:
        t0 = time.perf_counter()
        oracle.ll_gmp(p, k0)
        t1 = time.perf_counter()
        oracle.ll_gmp(p, k1)
        t2 = time.perf_counter()
        kind, call = "port", "oracle GMP restatement"
    else:
        t0 = time.perf_counter()
        ref.gmp_res64_after(p, k0)
        t1 = time.perf_counter()
        ref.gmp_res64_after(p, k1)
        t2 = time.perf_counter()
        kind, call = "reference", "reference gmp_res64_after"
    per = ((t2 - t1) - (t1 - t0)) / (k1 - k0)
    return {"value": round(per * 1e6, 1), "unit": "us/iteration", "cores": 1, "kind": kind,
            "sample": f"{call}(p={p}, {k1}) - ({k0}): {k1 - k0} full-size squarings of {what}"}


def cpu_baseline_big(threads):
    """Reference CPU time per Lucas-Lehmer squaring at p = 136,279,841, from the reference's own
    squaring micro-benchmark bench_square(bits, iters, depth) (lucaslehmer.cpp:181-205; GMP mpz
    square of a p-bit number, plain and with the reference's 9-thread Karatsuba split), compiled
    unchanged into oracle/_ref. The best of the two is the reported value."""
    from oracle import oracle
    ref = oracle.reference_module()
    if ref is None:  # the oracle's GMP restatement: one full-size squaring by difference
        t0 = time.perf_counter()
        oracle.ll_gmp(BIG_P, 27)
        t1 = time.perf_counter()
        oracle.ll_gmp(BIG_P, 29)
        t2 = time.perf_counter()
        per = ((t2 - t1) - (t1 - t0)) / 2.0
        return {"value": round(per * 1e6, 1), "unit": "us/iteration", "cores": 1, "kind": "port",
                "sample": "oracle GMP restatement, p=136,279,841, (t(29) - t(27)) / 2 squarings"}
    plain = ref.bench_square(BIG_P, 2, 0)
    depth = 2 if threads >= 9 else (1 if threads >= 3 else 0)
    split = ref.bench_square(BIG_P, 2, depth) if depth else float("inf")
    best = min(plain, split)
    return {"value": round(best * 1e6, 1), "unit": "us/iteration",
            "cores": {0: 1, 1: 3, 2: 9}[depth] if best == split else 1, "kind": "reference",
            "plain_1core_us": round(plain * 1e6, 1),
            "split_us": None if split == float("inf") else round(split * 1e6, 1), "split_depth": depth,
            "sample": "reference bench_square(136279841, iters=2, depth 0 and 2): seconds per "
                      "squaring of a 136,279,841-bit number (GMP; depth 2 = the reference's 9-thread "
                      "Karatsuba split), the mod 2^p-1 shift-and-add (~1% of a squaring) not included"}


# Published wall time of the reference's FFT engine (FFTW3) over every prime p <= 100001 on a Xeon
# w5-3435X with 32 threads (reference README.md:96,127-128): the yardstick of the range target.
PUBLISHED_FFT_RANGE = {"wall_s": 442.5, "threads": 32, "host": "Xeon w5-3435X (16C/32T)",
                       "tests_per_s": round(9592 / 442.5, 2), "source": "reference README.md:96,127-128"}


def _range_sample(threads, budget_s, cost_per_1e5):
    """Every k-th prime p <= 100001 (offset k/2), k the smallest power of two >= 64 whose sample
    fits the budget on `threads` threads (a test's cost grows as ~p^2.3)."""
    ps = sieve(2, RANGE_HI)
    k = 64
    est = lambda kk: sum((p / 1e5) ** 2.3 * cost_per_1e5 for p in ps[::kk]) / threads
    while est(k) > budget_s and k < 4096:
        k *= 2
    return ps, k, ps[k // 2::k]


def _time_sample(run, sample, threads):
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(run, sorted(sample, reverse=True)))
    return time.perf_counter() - t0


def cpu_baseline_range(threads, budget_s=20.0):
    """The reference's CPU engines (oracle/_ref: its lucaslehmer.cpp compiled unchanged) on a
    stratified sample of the range, all host threads: the GMP engine (lucas_lehmer_res,
    lucaslehmer.cpp:29-58) as the reported value, and the FFT engine (lucas_lehmer_fft_res,
    lucaslehmer.cpp:257-335) beside it. FFTW3 is not installed, so the FFT engine runs its own
    code over the oracle's radix-2 FFT behind FFTW's plan API, several times slower than FFTW;
    the published FFTW figure is quoted next to it."""
    from oracle import oracle
    ref = oracle.reference_module()
    kind = "reference" if ref else "port"
    ps, k, sample = _range_sample(threads, budget_s, 9.0)
    run = (lambda p: ref.lucas_lehmer_res(p)) if ref else (lambda p: oracle.ll_gmp(p)[:2])
    wall = _time_sample(run, sample, threads)
    out = {"value": round(len(ps) / (wall * k), 4), "unit": "tests/s", "cores": threads, "kind": kind,
           "sample": f"reference GMP engine (lucas_lehmer_res) on every {k}th prime p<=100001 "
                     f"({len(sample)} tests, {wall:.1f} s wall on {threads} threads); full-range wall "
                     f"extrapolated as sample wall x {k}"}
    if ref:
        ps, kf, fs = _range_sample(threads, budget_s, 25.0)
        wf = _time_sample(lambda p: ref.lucas_lehmer_fft_res(p), fs, threads)
        out["fft_engine"] = {
            "value": round(len(ps) / (wf * kf), 4), "unit": "tests/s", "cores": threads,
            "kind": "reference code over a substitute FFT",
            "sample": f"reference FFT engine (lucas_lehmer_fft_res) on every {kf}th prime p<=100001 "
                      f"({len(fs)} tests, {wf:.1f} s wall on {threads} threads), extrapolated x {kf}; "
                      "FFTW3 is absent, so its FFT calls run the oracle's radix-2 FFT (not FFTW)"}
    out["fft_engine_published"] = PUBLISHED_FFT_RANGE
    return out


REF_GPU_DIR = os.path.join(ROOT, "oracle", "_ref", "gpu")
_REF_GPU_CODE = r"""
import json, sys, time
sys.path.insert(0, sys.argv[1])
import lucaslehmer_cuda as ref
ps = json.loads(sys.argv[2])
ref.lucas_lehmer_batch(ps[:2])  # context, tables
t0 = time.perf_counter()
out = ref.lucas_lehmer_batch(ps)
wall = time.perf_counter() - t0
print(json.dumps({"wall": wall, "rows": [[p, bool(r), s, res] for p, r, s, res in out]}))
"""


def reference_gpu_range(every=8, timeout=600):
    """The reference's own GPU engine (its cuda/ll_ntt.cu compiled unchanged for sm_100a into
    oracle/_ref/gpu/: one block per exponent, radix-2 Goldilocks NTT in shared memory) on every
    `every`-th prime p <= 100001 on this GPU, in a subprocess (its module name is the product's).
    Exponents below 64 are not taken by that kernel (the driver runs them on the CPU); the rest are
    timed wall-clock around its lucas_lehmer_batch and their res64 checked against the golden."""
    if not os.path.exists(REF_GPU_DIR):
        return {"unavailable": "oracle/_ref/gpu not built (needs the reference's sources at build time)"}
    ps = [p for p in sieve(2, RANGE_HI) if p >= 64]
    sample = ps[every // 2::every]
    r = subprocess.run([sys.executable, "-c", _REF_GPU_CODE, REF_GPU_DIR, json.dumps(sample)],
                       capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        return {"unavailable": "reference GPU engine failed: " + (r.stderr.strip().splitlines() or ["?"])[-1][:200]}
    doc = json.loads(r.stdout.strip().splitlines()[-1])
    gold = {}
    for line in open(os.path.join(ROOT, "tests", "golden", "range_100001.csv")):
        if not line.startswith("#"):
            f = line.strip().split(",")
            gold[int(f[0])] = int(f[2], 16)
    bad = [p for p, isp, sec, res in doc["rows"] if sec >= 0 and res != gold[p]]
    taken = sum(1 for row in doc["rows"] if row[2] >= 0)
    full = len(ps) / len(sample)
    return {"value": round(len(sample) / doc["wall"], 3), "unit": "tests/s",
            "sample": f"every {every}th prime 64 <= p <= 100001 ({len(sample)} tests, {taken} taken by the kernel), "
                      f"{doc['wall']:.2f} s wall around lucas_lehmer_batch; the full range is ~{full:.1f}x the sample",
            "res64_mismatches": len(bad), "build": "reference cuda/ll_ntt.cu unchanged, nvcc -O3 sm_100a"}


def cpu_baseline_big_fft():
    """The reference's FFT engine (oracle/_ref) per squaring at p = 136,279,841, N = 2^23:
    fft_res64_after(p, 3) - fft_res64_after(p, 1), one thread, over the substitute FFT."""
    from oracle import oracle
    ref = oracle.reference_module()
    if ref is None:
        return None
    ref.fft_res64_after(BIG_P, 1)  # planning and tables of this length warmed
    t0 = time.perf_counter()
    ref.fft_res64_after(BIG_P, 1)
    t1 = time.perf_counter()
    ref.fft_res64_after(BIG_P, 3)
    t2 = time.perf_counter()
    per = ((t2 - t1) - (t1 - t0)) / 2.0
    return {"value": round(per * 1e6, 1), "unit": "us/iteration", "cores": 1,
            "kind": "reference code over a substitute FFT",
            "sample": "reference fft_res64_after(136279841, 3) - (136279841, 1): 2 squarings at N = 8,388,608; "
                      "FFTW3 is absent, so its FFT calls run the oracle's radix-2 FFT (not FFTW)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", choices=("big", "range", "single", "sweep"), default="big")
    ap.add_argument("--engine", choices=("fp64", "ntt"), default="fp64",
                    help="engine of the big workload; the reported engine of single and sweep")
    ap.add_argument("--sweep-iters", type=int, default=100000, help="sweep: FP64 squarings timed per prime")
    ap.add_argument("--sweep-ntt-iters", type=int, default=20000, help="sweep: NTT squarings timed per prime")
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="range: leave out the timing of the reference's own GPU engine")
    ap.add_argument("--no-range", action="store_true",
                    help="big: leave out the range sub-record (the other half of the metric)")
    ap.add_argument("--range-lengths", choices=("tuned", "rule"), default="tuned",
                    help="range: autotune the whole-test lengths (default) or keep the bits-per-digit "
                         "rule's (for profiler runs)")
    ap.add_argument("--split", default="",
                    help="big, FP64: the two-pass split 'log2 row length,rows per block' instead of the "
                         "autotuner's choice (e.g. 10,8)")
    args = ap.parse_args()
    threads = os.cpu_count() or 1
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return 0
        t0 = time.perf_counter()
        vals = []
        # the reference's CPU engine keeps no state between steps: warm-up steps are not repeated
        for _ in range(args.steps):
            if args.workload == "range":
                vals.append(cpu_baseline_range(threads, budget_s=15.0))
            elif args.workload == "single":
                vals.append(cpu_baseline_interim(SINGLE_P, 40, 2040, "a 1,257,787-bit residue"))
            elif args.workload == "sweep":
                vals.append(cpu_baseline_interim(22685363, 30, 130, "a 22,685,363-bit residue"))
            else:
                vals.append(cpu_baseline_big(threads))
        v = statistics.median(x["value"] for x in vals)
        extra = {}
        if args.workload == "big":
            vals[-1]["fft_engine"] = cpu_baseline_big_fft()
            if not args.no_range:  # the other half of the metric, sampled once
                extra["range"] = cpu_baseline_range(threads, budget_s=15.0)
        if args.workload == "range":
            metric, unit, hib, scaling = METRIC_RANGE, "tests/s", True, "strong"
            cfg = {"workload": "range p<=100001 (9592 LL tests)"}
        elif args.workload == "single":
            metric, unit, hib, scaling = METRIC_SINGLE, "us/iteration", False, "weak"
            cfg = {"workload": "p=1,257,787, one Lucas-Lehmer squaring (reference GMP engine)"}
        elif args.workload == "sweep":
            metric, unit, hib, scaling = METRIC_SWEEP, "us/iteration", False, "weak"
            cfg = {"workload": "p=22,685,363 (median sweep prime), one Lucas-Lehmer squaring (reference GMP engine)"}
        else:
            metric, unit, hib, scaling = METRIC_BIG, "us/iteration", False, "weak"
            cfg = {"workload": "p=136,279,841, one Lucas-Lehmer squaring (reference GMP engine)"}
        line = {"metric": metric, "value": v, "unit": unit, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": hib,
                "scaling": scaling, "vs_baseline": None, "dtype": "int64 (GMP limbs)", "data": "synthetic",
                "config": cfg, "impl": "reference", "cpu_baseline": vals[-1],
                "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "ms_per_step": round(1e3 * (time.perf_counter() - t0) / max(1, args.steps), 1)}
        line.update(extra)
        print(json.dumps(line))
        return 0
    rank, world, local = dist_setup(args.gpus)
    bench = {"range": bench_range, "single": bench_single, "sweep": bench_sweep}.get(args.workload, bench_big)
    line = bench(args, rank, world)
    rng = None
    if args.workload == "big" and not args.no_range:
        # the other half of the metric: every prime p <= 100001, one timed step after one warm-up
        rng = bench_range(argparse.Namespace(**{**vars(args), "steps": 1, "warmup": 1}), rank, world)
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:
            if args.workload == "range":
                line["cpu_baseline"] = cpu_baseline_range(threads)
            elif args.workload == "single":
                line["cpu_baseline"] = cpu_baseline_interim(SINGLE_P, 40, 2040, "a 1,257,787-bit residue")
            elif args.workload == "sweep":
                line["cpu_baseline"] = cpu_baseline_interim(22685363, 30, 130, "a 22,685,363-bit residue")
            else:
                line["cpu_baseline"] = cpu_baseline_big(threads)
                line["cpu_baseline"]["fft_engine"] = cpu_baseline_big_fft()
                if rng is not None:
                    rng["cpu_baseline"] = cpu_baseline_range(threads)
        if rng is not None:
            for k in ("n_gpus", "steps", "warmup", "higher_is_better", "scaling", "vs_baseline", "dtype"):
                rng.pop(k, None)
            line["range"] = rng
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
