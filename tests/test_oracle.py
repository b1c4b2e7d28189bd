"""The oracle (CPU restatement of the reference's path) pinned against the reference's own golden
vectors: the hit set of known Mersenne exponents, the reference GMP engine's res64 values (from the
reference compiled unchanged, tests/golden/appendix.json), the reference README's published
interim residue, and the reference's own cross-engine checks (tests/test_lucaslehmer.py). CPU only."""
import os
import random

import pytest

from conftest import GOLDEN, KNOWN, load_json, load_range, known_exponents


def test_known_mersenne_exponents_gmp(oracle):
    # reference tests/test_lucaslehmer.py:11-13
    found = [p for p in oracle.primes(2, 4423) if oracle.ll_gmp(p)[0]]
    assert found == KNOWN


def test_non_mersenne(oracle):
    # reference tests/test_lucaslehmer.py:15-16
    assert not oracle.ll_gmp(11)[0] and not oracle.ll_gmp(23)[0] and not oracle.ll_gmp(4)[0]


def test_primes_sieve(oracle):
    # reference tests/test_lucaslehmer.py:5-9
    assert len(oracle.primes(2, 10001)) == 1229
    assert oracle.primes(0, 1) == [] and oracle.primes(2, 2) == [2] and oracle.primes(10, 20) == [11, 13, 17, 19]
    assert len(oracle.primes(2, 100001)) == 9592


def test_known_list_matches_sieve(oracle):
    ks = known_exponents()
    assert len(ks) == 52 and ks[0] == 2 and ks[-1] == 136279841
    assert [p for p in ks if p <= 4423] == KNOWN


def test_full_res64_vs_reference_goldens(oracle):
    # reference tests/test_lucaslehmer.py:49-53, values from the reference's lucas_lehmer_res
    g = load_json("appendix.json")
    for row in g["full"]:
        v, r, _ = oracle.ll_gmp(row["p"])
        assert v == row["is_prime"] and f"{r:016x}" == row["res64"]
        assert (r == 0) == v


@pytest.mark.parametrize("p,k", [(1257787, 240), (1257787, 1000), (22000007, 60), (136279841, 34)])
def test_interim_res64_vs_reference_goldens(oracle, p, k):
    g = {(d["p"], d["k"]): d["res64"] for d in load_json("appendix.json")["after"]}
    _, r, _ = oracle.ll_gmp(p, k)
    assert f"{r:016x}" == g[(p, k)]


def test_readme_published_residue_is_in_goldens():
    # README.md:204-206: prime95, the reference GMP engine and the reference FFT engine agree
    g = {(d["p"], d["k"]): d["res64"] for d in load_json("appendix.json")["after"]}
    assert g[(3021377, 20000)] == "ce811e3772129824"


def test_sweep_primes_are_the_seeded_sample(oracle):
    g = load_json("appendix.json")
    ps = oracle.primes(20000000, 25000000)
    assert sorted(random.Random(0).sample(ps, 8)) == g["sweep_primes"]
    assert len(g["sweep_primes"]) == 8


def test_range_golden_sample(oracle):
    rows = load_range()
    assert len(rows) == 9592
    assert sorted(p for p, (v, _, _) in rows.items() if v) == [p for p in known_exponents() if p <= 100001]
    rng = random.Random(7)
    for p in rng.sample([p for p in rows if p <= 20000], 25) + [4423, 4253, 9689, 19937]:
        v, r, words = oracle.ll_gmp(p)
        assert (v, r, oracle.residue_hash(words)) == rows[p], p


def test_trace_golden_consistent():
    t = load_json("trace_1257787.json")
    g = {(d["p"], d["k"]): d["res64"] for d in load_json("appendix.json")["after"]}
    assert t["res64"][0] == g[(1257787, 10000)]
    assert t["res64_after_1000"] == g[(1257787, 1000)]
    assert len(t["res64"]) == (1257787 - 2) // 10000


def test_ibdwt_restatement_matches_gmp(oracle):
    # reference tests/test_lucaslehmer.py:32-36 (FFT engine == GMP; fft_info(9689))
    for p in oracle.primes(4425, 6000)[::7] + [4423, 9689]:
        v, r, err, _, _ = oracle.ibdwt(p)
        g = oracle.ll_gmp(p)
        assert v == int(g[0]) and r == g[1], p
        assert err < 0.05
    assert oracle.fft_length(9689) == 640 and 9689 / 640 <= 18


def test_ibdwt_interim_digits_rebuild(oracle):
    p = 20011
    for k in (1, 2, 37, 500):
        v, r, err, words, digits = oracle.ibdwt(p, iters=k, want_digits=True)
        g = oracle.ll_gmp(p, k)
        assert words == g[2]
        z, r2, w2 = oracle.rebuild(p, len(digits), digits)
        assert w2 == g[2]


def test_goldilocks_field_ops(oracle):
    q = 2**64 - 2**32 + 1
    rng = random.Random(3)
    for _ in range(200):
        a, b = rng.randrange(q), rng.randrange(q)
        L = oracle.lib()
        assert L.orc_gl_mul(a, b) == a * b % q
        assert L.orc_gl_add(a, b) == (a + b) % q
        assert L.orc_gl_sub(a, b) == (a - b) % q
    for logn in (6, 10, 16, 20, 23):
        N = 1 << logn
        om, r2, inv = oracle.ntt_tables(N)
        assert pow(om, N, q) == 1 and pow(om, N // 2, q) == q - 1
        assert pow(r2, N, q) == 2
        assert inv * N % q == 1


def test_ntt_restatement_matches_gmp(oracle):
    # reference cuda/ll_ntt.cu:172-180 length rule and tests/test_lucaslehmer.py:39-46
    L = oracle.lib()
    assert L.orc_ntt_length(127) == 64 and L.orc_ntt_max_bits(64) == 28 and L.orc_ntt_max_bits(8192) == 25
    for p in (521, 607, 1279, 2203, 2281, 1223, 4423):
        v, r, w, _ = oracle.ntt(p)
        g = oracle.ll_gmp(p)
        assert (bool(v), r, w) == (g[0], g[1], g[2]), p


def test_reference_module_agrees_when_present(oracle):
    ref = oracle.reference_module()
    if ref is None:
        pytest.skip("reference build (oracle/_ref) not present")
    for p in (4425, 9689, 20011, 521, 11213):
        assert ref.lucas_lehmer_res(p) == oracle.ll_gmp(p)[:2]
        assert ref.lucas_lehmer_fft_res(p) == oracle.ll_gmp(p)[:2]
    assert ref.gmp_res64_after(1257787, 240) == oracle.ll_gmp(1257787, 240)[1]
