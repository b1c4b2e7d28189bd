"""Parity of the CUDA path with the oracle, through the C-ABI (libllgpu.so via ctypes).

Bit-exact integer results: full residues (every limb) against the oracle's GMP restatement and
the committed golden fingerprints; the word path (p < 64); every power-of-two length of the
whole-test kernel; interim residues; the round-off escalation path."""
import os
import random

import pytest

from conftest import GOLDEN, load_range

pytestmark = pytest.mark.gpu


def test_word_path_all_small_exponents(gpu, oracle):
    """p < 256 runs on the exact multi-limb kernel: every exponent, full residue."""
    for p in range(2, 256):
        r = gpu.run(p, want_words=True)
        v, res, words = oracle.ll_gmp(p)
        assert (bool(r["is_zero"]), r["res64"]) == (v, res), p
        if p >= 3 and p % 2:
            assert r["words"] == words


@pytest.mark.parametrize("logn", range(5, 14))
def test_every_length_full_residue(gpu, oracle, logn):
    n = 1 << logn
    rng = random.Random(logn)
    lo = max(256, n * ((logn + 5) // 2))  # the length's bits-per-digit floor
    ps = [p for p in oracle.primes(lo, min(18 * n, 30000)) if p % 2]
    for p in rng.sample(ps, min(4, len(ps))):
        r = gpu.run(p, n=n, want_words=True)
        v, res, words = oracle.ll_gmp(p)
        assert r["status"] == 0 and r["n"] == n
        assert r["words"] == words, (p, n)
        assert bool(r["is_zero"]) == v and r["max_err"] < 0.4


@pytest.mark.parametrize("p,k", [(127, 1), (4423, 2), (9689, 3), (20011, 17), (44497, 1000), (100003, 123)])
def test_interim_full_residue(gpu, oracle, p, k):
    r = gpu.run(p, iters=k, want_words=True)
    assert r["iters"] == k
    assert r["words"] == oracle.ll_gmp(p, k)[2]


def test_all_primes_to_10001_full_residues(gpu, oracle):
    """Config: every prime p <= 10001 (1229 exponents, 22 hits), full residues bit-exact."""
    rows = load_range()
    ps = [p for p in oracle.primes(2, 10001)]
    out = gpu.run_batch(ps, want_words=True)
    hits = []
    for p, r in zip(ps, out):
        v, res, h = rows[p]
        assert r["status"] == 0
        assert (bool(r["is_zero"]), r["res64"], oracle.residue_hash(r["words"])) == (v, res, h), p
        if r["is_zero"]:
            hits.append(p)
    assert len(hits) == 22


def test_batch_matches_single(gpu):
    ps = [1279, 2203, 4421, 9941, 11213, 19937, 21701, 23209]
    b = gpu.run_batch(ps, iters=500)
    for p, rb in zip(ps, b):
        rs = gpu.run(p, iters=500)
        assert rb["res64"] == rs["res64"] and rb["n"] == rs["n"]


@pytest.mark.parametrize("p,n", [(27611, 1024), (138239, 5120)])
def test_roundoff_escalation_stays_exact(gpu, oracle, p, n):
    """Force a length far too short (27 bits per digit: the convolution outgrows FP64's 53 bits),
    a power of two and a 5 x 2^k length: the kernel must abort on round-off, the host must redo it
    at a longer length on the GPU, and the residue must still be exact."""
    r = gpu.run(p, iters=300, n=n, want_words=True)
    assert r["status"] == 0 and r["escalations"] >= 1 and r["n"] > n
    assert r["words"] == oracle.ll_gmp(p, 300)[2]


def test_unsupported_exponent_is_an_error(gpu):
    with pytest.raises(gpu.LlgError):
        gpu.run(10**12 + 39)


def test_trivial_exponents(gpu):
    assert gpu.run(2)["is_zero"] == 1
    assert gpu.run(4)["is_zero"] == 0
    assert gpu.run(1)["is_zero"] == 0
    assert gpu.run(0)["is_zero"] == 0


# ---- the exact Goldilocks NTT engine ----------------------------------------------------------

@pytest.mark.parametrize("logn", range(6, 14))
def test_ntt_every_length_full_residue(gpu, oracle, logn):
    """Every NTT length at bits per digit spanning the exactness bound ceil(p/N) <= (63-log2 N)/2."""
    n = 1 << logn
    hi = ((63 - logn) // 2) * n
    lo = max(256, n * ((logn + 12 + 3) // 4))
    rng = random.Random(100 + logn)
    ps = [p for p in oracle.primes(lo, min(hi, 40000)) if p % 2]
    picks = rng.sample(ps, min(3, len(ps))) + ([max(ps)] if ps else [])
    for p in picks:
        r = gpu.run(p, engine="ntt", n=n, want_words=True)
        assert r["status"] == 0 and r["n"] == n
        assert r["words"] == oracle.ll_gmp(p)[2], (p, n)


def test_ntt_length_rule_matches_reference():
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    from oracle import oracle
    # the reference's ntt_length (cuda/ll_ntt.cu:176-180), where its own kernel can run (p >= 256)
    for p in (521, 1279, 4423, 9689, 44497, 100003, 204799):
        assert llgpu.ntt_length(p) == oracle.lib().orc_ntt_length(p), p


def test_ntt_matches_fp64_and_oracle_batch(gpu, oracle):
    ps = [p for p in oracle.primes(320, 12000)][::5]  # the NTT takes p >= 5 * 64 (bits-per-digit floor)
    a = gpu.run_batch(ps, engine="ntt", want_words=True)
    b = gpu.run_batch(ps, engine="fp64", want_words=True)
    for p, ra, rb in zip(ps, a, b):
        assert ra["status"] == 0 and ra["words"] == rb["words"], p
    for p, ra in list(zip(ps, a))[::10]:
        assert ra["words"] == oracle.ll_gmp(p)[2], p


def test_ntt_interim_residue(gpu, oracle):
    for p, k in ((4423, 3), (86243, 1000), (204791, 77)):
        r = gpu.run(p, iters=k, engine="ntt", want_words=True)
        assert r["words"] == oracle.ll_gmp(p, k)[2]


# ---- the non-power-of-two whole-test lengths (3 x 2^k, 5 x 2^k) --------------------------------

@pytest.mark.parametrize("n", [3072, 5120, 6144, 10240, 12288])
def test_mixed_length_full_residue(gpu, oracle, n):
    """Every {3,5} x 2^k length, exponents from the bits-per-digit floor to 18 bits per digit,
    full residues (every limb) after all p - 2 squarings or an interim k."""
    rng = random.Random(n)
    lo = n * ((n.bit_length() + 4 + 1) // 2)
    ps = [p for p in oracle.primes(lo, min(18 * n, 230000)) if p % 2]
    picks = sorted(rng.sample(ps, 3)) + [max(ps)]
    for p in picks:
        k = 0 if p < 60000 else 3000  # full tests where the oracle finishes in seconds
        r = gpu.run(p, n=n, iters=k, want_words=True)
        assert r["status"] == 0 and r["n"] == n, (p, n, r)
        assert r["words"] == oracle.ll_gmp(p, k)[2], (p, n)
        assert r["max_err"] < 0.4


def test_mixed_lengths_in_batch(gpu, oracle):
    """A batch mixing power-of-two and {3,5} x 2^k buckets, results in input order."""
    ps = [44497, 40009, 80021, 9689, 99991, 86243, 150001, 4423]
    rs = gpu.run_batch(ps, iters=2000, want_words=True)
    lengths = {r["p"]: r["n"] for r in rs}
    assert lengths[44497] == 3072 and lengths[80021] == 5120 and lengths[99991] == 6144
    for p, r in zip(ps, rs):
        assert r["p"] == p and r["words"] == oracle.ll_gmp(p, 2000)[2], p


def test_mixed_length_known_primes(gpu):
    """The Mersenne exponents whose lengths are 3 x 2^10 and 5 x 2^10 (full tests: residue zero)."""
    for p in (44497, 86243):
        r = gpu.run(p)
        assert r["n"] in (3072, 5120) and r["is_zero"] == 1 and r["status"] == 0, r


def test_all_primes_to_100001_full_residues(gpu, oracle):
    """Config: every prime p <= 100001 (9592 exponents, 28 hits) in one batch, the mix of lengths
    the engine picks (power-of-two and {3,5} x 2^k): every full residue's fingerprint equals the
    oracle's (tests/golden/range_100001.csv), and the hit set is the known list."""
    from conftest import known_exponents
    rows = load_range()
    ps = oracle.primes(2, 100001)
    out = gpu.run_batch(ps, want_words=True)
    hits = []
    for p, r in zip(ps, out):
        v, res, h = rows[p]
        assert r["status"] == 0, p
        assert (bool(r["is_zero"]), r["res64"], oracle.residue_hash(r["words"])) == (v, res, h), p
        if r["is_zero"]:
            hits.append(p)
    assert hits == [p for p in known_exponents() if p <= 100001]


def test_range_autotuner_keeps_residues_exact(gpu):
    """llgpu.autotune_range times each bucket's candidate lengths and puts the fastest in force;
    with its choices every prime p <= 10001 still has the reference's residue, and clearing them
    restores the rule's lengths."""
    from conftest import load_range
    gold = load_range()
    out = gpu.autotune_range(hi=10001, iters=200, tests=148, save=False)
    try:
        assert out and all(best >= n for n, (best, _) in out.items())
        ps = [p for p in sorted(gold) if p <= 10001]
        res = gpu.run_batch(ps)
        assert all((bool(r["is_zero"]), r["res64"]) == gold[r["p"]][:2] for r in res)
    finally:
        for n in out:
            gpu.set_length_choice(n, 0)
    assert all(gpu.get_length_choice(n) == n for n in out)
