"""The reference's own test suite (tests/test_lucaslehmer.py), run against this engine's
`lucaslehmer` / `lucaslehmer_cuda` modules on the GPU, plus the driver's exit-status contract."""
import os
import subprocess
import sys

import pytest

from conftest import KNOWN, PKG, ROOT, load_json

pytestmark = pytest.mark.gpu


def test_known_mersenne_exponents(ll):
    # reference tests/test_lucaslehmer.py:11-13
    found = [p for p in ll.primes(2, 4423) if ll.lucas_lehmer(p)]
    assert found == KNOWN


def test_non_mersenne(ll):
    # reference tests/test_lucaslehmer.py:15-16
    assert not ll.lucas_lehmer(11) and not ll.lucas_lehmer(23) and not ll.lucas_lehmer(4)


def test_compat_class(ll):
    # reference tests/test_lucaslehmer.py:21-23
    c = ll.LucasLehmer()
    out = []
    assert c.sa_lucaslehmer(31, 4) is True and c.sa_getListOfPrimes(out, 2, 10) is True and out == [2, 3, 5, 7]


def test_split_matches_plain(ll):
    # reference tests/test_lucaslehmer.py:26-29
    for d in (1, 2):
        assert [p for p in ll.primes(2, 4423) if ll.lucas_lehmer_split(p, d)] == KNOWN
        assert not ll.lucas_lehmer_split(4425, d)


def test_fft_engine_matches_known_and_gmp(ll, oracle):
    # reference tests/test_lucaslehmer.py:32-36; the GMP side is the oracle
    assert [p for p in ll.primes(2, 4423) if ll.lucas_lehmer_fft(p)] == KNOWN
    assert all(ll.lucas_lehmer_fft(p) == oracle.ll_gmp(p)[0] for p in ll.primes(4425, 6000))
    n, bpw, err = ll.fft_info(9689)
    assert ll.lucas_lehmer_fft(9689) and err < 0.05 and bpw <= 18


def test_cuda_engine(ll, lc, oracle):
    # reference tests/test_lucaslehmer.py:39-46 (here the module is always built)
    res = {p: r for p, r, s, res64 in lc.lucas_lehmer_batch(ll.primes(2, 4423)) if s >= 0}
    assert sorted(p for p, r in res.items() if r) == [p for p in KNOWN if p in res]
    assert all(res[p] == oracle.ll_gmp(p)[0] for p in res)
    name, sms, mem = lc.device_info()
    assert sms > 0 and mem > 0 and lc.max_exponent() > 0


def test_cuda_engine_ntt(ll, lc, oracle):
    """lucaslehmer_cuda's own engine (cuda/ll_ntt.cu) is the exact NTT: the same contract."""
    res = {p: r for p, r, s, res64 in lc.lucas_lehmer_batch(ll.primes(2, 4423), engine="ntt") if s >= 0}
    assert sorted(p for p, r in res.items() if r) == [p for p in KNOWN if p in res]
    assert all(res[p] == oracle.ll_gmp(p)[0] for p in res)


def test_res64_agrees_across_engines(ll):
    # reference tests/test_lucaslehmer.py:49-53, against the reference's own values
    gold = {row["p"]: (row["is_prime"], int(row["res64"], 16)) for row in load_json("appendix.json")["full"]}
    for p in (4425, 9689, 20011):
        g = ll.lucas_lehmer_res(p)
        f = ll.lucas_lehmer_fft_res(p)
        s = ll.lucas_lehmer_split_res(p, 1)
        assert g == f == s == gold[p]
        assert (g[1] == 0) == g[0]


def test_interim_residue_api(ll, oracle):
    for p, k in ((4423, 1), (4423, 100), (20011, 7), (86243, 1000)):
        want = oracle.ll_gmp(p, k)[1]
        r, err = ll.fft_res64_after(p, k)
        assert r == want and err < 0.4
        assert ll.gmp_res64_after(p, k) == want


def test_driver_runs_unchanged(tmp_path):
    """The reference driver's contract: the hit set matches the known list and the exit status is 0.
    The driver itself is not shipped here; this runs its documented call sequence for --engine fft
    and --engine cuda through the modules (test_one + the cuda chunking)."""
    code = r'''
import sys
sys.path.insert(0, sys.argv[1])
import lucaslehmer as ll, lucaslehmer_cuda as lc
ps = ll.primes(2, 10001)
hits = [p for p in ps if ll.lucas_lehmer_fft_res(p)[0]]
chunks = []
for p in sorted(ps):
    N = lc.ntt_length(p) if p >= 64 else 0
    if chunks and chunks[-1][0] == N and len(chunks[-1][1]) < 2048: chunks[-1][1].append(p)
    else: chunks.append((N, [p]))
cuda_hits = []
for N, group in chunks:
    res = {p: (r, dt, rs) for p, r, dt, rs in lc.lucas_lehmer_batch(group)} if N else {}
    for p in group:
        if p in res and res[p][1] >= 0: r = res[p][0]
        else: r = ll.lucas_lehmer_fft_res(p)[0]
        if r: cuda_hits.append(p)
known = [2, 3, 5, 7, 13, 17, 19, 31, 61, 89, 107, 127, 521, 607, 1279, 2203, 2281, 3217, 4253, 4423, 9689, 9941]
sys.exit(0 if hits == known and sorted(cuda_hits) == known else 2)
'''
    r = subprocess.run([sys.executable, "-c", code, PKG], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


def test_concurrent_callers_share_batches(gpu, oracle):
    """Single-exponent calls from many host threads at once (the driver's thread pool) are pooled
    into shared batches: every caller gets its own exact result, whether it asked for a full test or
    an interim residue, for its words or not, on either engine."""
    from concurrent.futures import ThreadPoolExecutor
    from conftest import load_range
    gold = load_range()
    ps = [p for p in range(3, 6000) if p in gold]
    jobs = []
    for i, p in enumerate(ps):
        if i % 7 == 3 and gpu.ntt_length(p):
            jobs.append((p, 0, "ntt", False))
        elif i % 11 == 5 and p > 300:
            jobs.append((p, 50, "fp64", True))
        else:
            jobs.append((p, 0, "fp64", False))

    def one(job):
        p, k, engine, words = job
        return job, gpu.run(p, iters=k, engine=engine, want_words=words)

    with ThreadPoolExecutor(32) as ex:
        results = list(ex.map(one, jobs))
    for (p, k, engine, words), r in results:
        assert r["status"] == 0, (p, engine)
        if k == 0:
            assert (bool(r["is_zero"]), r["res64"]) == gold[p][:2], (p, engine)
        else:
            want = oracle.ll_gmp(p, k)
            assert r["res64"] == want[1] and r["words"] == want[2], p
