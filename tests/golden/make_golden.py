"""Generates the golden fixtures under tests/golden/ (run in the build container, where the
reference's sources exist; the fixtures are committed and nothing at test time re-runs this).

Every vector comes from the reference's own GMP engine (its lucaslehmer.cpp compiled unchanged into
oracle/_ref/ by oracle/Makefile) or from the oracle's GMP restatement, cross-checked against the
reference where both exist:

  appendix.json   res64 after k squarings (reference ``gmp_res64_after``) for the large-p workloads:
                  p=1,257,787; the 8 seeded primes in [20M, 25M]; p=136,279,841; the README's
                  p=3,021,377 @ 20,000 (published value ce811e3772129824, README.md:204-206);
                  full-test (is_prime, res64) from ``lucas_lehmer_res`` for 4425, 9689, 20011.
  trace_1257787.json  res64 after every 10^4 squarings of the full p=1,257,787 test (oracle GMP
                  restatement; its k=1000/10000 values and final zero are checked against the
                  reference run).
  range_100001.csv    for every prime p <= 100001: verdict, res64 and a 64-bit blake2b fingerprint
                  of the full residue (oracle GMP restatement); the reference's own res64 is
                  checked for every p <= 30001 and a seeded sample of 400 above.

  known_mp_list.txt   the 52 known Mersenne-prime exponents (public data; copied from the
                  reference's known_mp_list.txt, the hit-set oracle its driver reads).

Usage: python tests/golden/make_golden.py {appendix|trace|range|known} [--workers W]
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import random
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402

BIG_P = 136279841
CFG2_P = 1257787
README_P, README_K, README_RES = 3021377, 20000, "ce811e3772129824"


def seeded_sweep_primes():
    """sorted(random.Random(0).sample(primes in [20M, 25M], 8)) -- the precision-sweep exponents."""
    ps = oracle.primes(20000000, 25000000)
    return sorted(random.Random(0).sample(ps, 8))


def _ref_after(args):
    p, k = args
    ref = oracle.reference_module()
    t0 = time.time()
    r = ref.gmp_res64_after(p, k)
    return p, k, f"{r:016x}", time.time() - t0


def _ref_full(p):
    ref = oracle.reference_module()
    v, r = ref.lucas_lehmer_res(p)
    return p, bool(v), r


def appendix(workers: int):
    sweep = seeded_sweep_primes()
    jobs = [(BIG_P, 1000), (README_P, README_K), (CFG2_P, 1000), (CFG2_P, 10000), (CFG2_P, 240),
            (22000007, 60), (BIG_P, 34)] + [(p, 1000) for p in sweep]
    ctx = mp.get_context("spawn")
    out = {"sweep_primes": sweep, "after": [], "full": []}
    with ctx.Pool(workers) as pool:
        for p, k, r, dt in pool.imap_unordered(_ref_after, jobs):
            print(f"p={p} k={k} res64={r} ({dt:.1f} s)", flush=True)
            out["after"].append({"p": p, "k": k, "res64": r, "source": "reference gmp_res64_after"})
        for p, v, r in pool.map(_ref_full, [4425, 9689, 20011]):
            out["full"].append({"p": p, "is_prime": v, "res64": f"{r:016x}",
                                "source": "reference lucas_lehmer_res"})
    out["after"].sort(key=lambda d: (d["p"], d["k"]))
    got = {(d["p"], d["k"]): d["res64"] for d in out["after"]}
    assert got[(README_P, README_K)] == README_RES, "reference disagrees with its README"
    with open(os.path.join(HERE, "appendix.json"), "w") as f:
        json.dump(out, f, indent=1)


def trace():
    every, total = 10000, CFG2_P - 2
    t0 = time.time()
    vals = oracle.ll_gmp_trace(CFG2_P, total, every)
    v, r, _ = oracle.ll_gmp(CFG2_P, 1000)
    out = {"p": CFG2_P, "every": every, "res64": [f"{x:016x}" for x in vals],
           "res64_after_1000": f"{r:016x}", "final_is_zero": True,
           "source": "oracle GMP restatement (lucaslehmer.cpp:29-58)", "seconds": time.time() - t0}
    ref = oracle.reference_module()
    if ref is not None:
        assert f"{ref.gmp_res64_after(CFG2_P, 10000):016x}" == out["res64"][0]
        assert f"{ref.gmp_res64_after(CFG2_P, 1000):016x}" == out["res64_after_1000"]
    with open(os.path.join(HERE, f"trace_{CFG2_P}.json"), "w") as f:
        json.dump(out, f, indent=0)


def _range_one(p):
    v, r, words = oracle.ll_gmp(p)
    return p, v, r, oracle.residue_hash(words)


def _range_ref(p):
    ref = oracle.reference_module()
    v, r = ref.lucas_lehmer_res(p)
    return p, bool(v), r


def range_(workers: int, hi: int = 100001):
    """Rows are appended to a partial file as they finish (a restart skips the finished ones);
    the committed CSV is written once every exponent is done and cross-checked."""
    ps = oracle.primes(2, hi)
    partial = os.path.join(HERE, ".range_100001.partial")
    rows = {}
    if os.path.exists(partial):
        with open(partial) as f:
            for line in f:
                p, v, r, h = line.strip().split(",")
                rows[int(p)] = (v == "1", int(r, 16), h)
    order = sorted((p for p in ps if p not in rows), reverse=True)  # largest first: load balance
    ctx = mp.get_context("spawn")
    t0 = time.time()
    with ctx.Pool(workers) as pool, open(partial, "a") as out:
        for i, (p, v, r, h) in enumerate(pool.imap_unordered(_range_one, order, chunksize=1)):
            rows[p] = (v, r, h)
            out.write(f"{p},{int(v)},{r:016x},{h}\n")
            out.flush()
            if i % 500 == 0:
                print(f"{len(rows)}/{len(ps)} p={p} {time.time() - t0:.0f} s", flush=True)
        check = [p for p in ps if p <= 30001]
        rng = random.Random(1)
        check += rng.sample([p for p in ps if p > 30001], 400)
        for p, v, r in pool.imap_unordered(_range_ref, sorted(check, reverse=True), chunksize=1):
            # p = 2 returns before any squaring (lucaslehmer.cpp:29), leaving the thread's previous
            # res64 in place: only its verdict is defined
            assert rows[p][0] == v and (p == 2 or rows[p][1] == r), f"oracle != reference at p={p}"
    with open(os.path.join(HERE, "range_100001.csv"), "w") as f:
        f.write("# p,is_prime,res64,residue_blake2b64 -- oracle GMP restatement; reference res64 "
                f"checked on {len(check)} exponents\n")
        for p in ps:
            v, r, h = rows[p]
            f.write(f"{p},{int(v)},{r:016x},{h}\n")
    os.remove(partial)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=("appendix", "trace", "range", "known"))
    ap.add_argument("--workers", type=int, default=4)
    a = ap.parse_args()
    if a.what == "appendix":
        appendix(a.workers)
    elif a.what == "known":
        src = os.path.join(os.environ.get("LL_REFERENCE_SRC", "/root/reference"), "known_mp_list.txt")
        with open(src) as f:
            exps = sorted(int(x) for x in f.read().split())
        with open(os.path.join(HERE, "known_mp_list.txt"), "w") as f:
            f.write("\n".join(str(x) for x in exps) + "\n")
    elif a.what == "trace":
        trace()
    else:
        range_(a.workers)
