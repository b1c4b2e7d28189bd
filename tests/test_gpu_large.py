"""Parity of the two-pass engine (lengths 2^14 .. 2^23, state in HBM) with the oracle and with the
reference's own golden residues, through the C-ABI.

Interim residues are compared in full (every limb) against the oracle's GMP restatement where the
oracle finishes in seconds, and as res64 against the reference's gmp_res64_after values
(tests/golden/appendix.json, trace_1257787.json) at the benchmark sizes."""
import pytest

from conftest import load_json

pytestmark = pytest.mark.gpu


def _after():
    return {(d["p"], d["k"]): int(d["res64"], 16) for d in load_json("appendix.json")["after"]}


@pytest.mark.parametrize("logn", range(14, 24))
def test_every_large_length_full_residue(gpu, oracle, logn):
    """Every supported two-pass length, a p at ~16.5 bits/digit, past the first wrap-around."""
    n = 1 << logn
    p = int(16.5 * n) | 1
    while any(p % d == 0 for d in (3, 5, 7, 11, 13)):
        p += 2
    k = p.bit_length() + 4  # s_k exceeds 2^p after ~log2(p) squarings: the reduction is exercised
    r = gpu.run(p, iters=k, n=n, want_words=True)
    assert r["status"] == 0 and r["n"] == n and r["iters"] == k
    assert r["words"] == oracle.ll_gmp(p, k)[2]
    assert r["max_err"] < 0.1


@pytest.mark.parametrize("p,k", [(1257787, 240), (1257787, 1000), (1257787, 10000)])
def test_config_p1257787_at_65536(gpu, p, k):
    """p = 1,257,787 at N = 65536 (19.19 bits/digit), res64 after k vs the reference GMP engine."""
    r = gpu.run(p, iters=k, n=65536)
    assert r["status"] == 0 and r["n"] == 65536
    assert r["res64"] == _after()[(p, k)]


def test_config_sweep_primes_1000(gpu):
    """The 8 seeded primes in [20M, 25M]: res64 after 1000 squarings vs the reference GMP engine.
    Length chosen at 19.5 bits/digit (2^20 where it fits, else 2^21), escalated on round-off."""
    g = load_json("appendix.json")
    after = _after()
    for p in g["sweep_primes"]:
        n = gpu.fft_length(p, 19.5)
        r = gpu.run(p, iters=1000, n=n)
        assert r["status"] == 0, p
        assert r["res64"] == after[(p, 1000)], p
        assert r["max_err"] <= 0.4


@pytest.mark.parametrize("k", [34, 1000])
def test_config_largest_p136279841(gpu, k):
    """p = 136,279,841 at N = 2^23 (16.25 bits/digit): res64 after k squarings vs the reference."""
    r = gpu.run(136279841, iters=k, n=1 << 23)
    assert r["status"] == 0 and r["n"] == 1 << 23
    assert r["res64"] == _after()[(136279841, k)]
    assert r["max_err"] < 0.4


def test_test_object_interim_and_errlog(gpu, oracle):
    """llg_test_*: start / iterate in pieces / read equals one run; the round-off log is filled."""
    p, n = 3021377, 1 << 18
    t = gpu.Test(p, n)
    t.start()
    t.iterate(999)
    mid = t.read()  # start did the first squaring; reading does not disturb the state
    assert mid["iters"] == 1000 and mid["res64"] == gpu.run(p, iters=1000, n=n)["res64"]
    t.iterate(1000)
    r = t.read(want_words=True)
    assert r["iters"] == 2000
    one = gpu.run(p, iters=2000, n=n, want_words=True)
    assert r["words"] == one["words"]
    log = t.errlog(2001)
    assert len(log) >= 2000 and max(log[1:2000]) > 0 and max(log) <= r["max_err"] + 1e-7
    t.close()


def test_readme_interim_residue(gpu):
    """README.md:204-206: res64 of p = 3,021,377 after 20,000 squarings is ce811e3772129824."""
    r = gpu.run(3021377, iters=20000)
    assert r["res64"] == 0xCE811E3772129824


def test_large_escalation_exact(gpu, oracle):
    """A length far too short for FP64 (27 bits/digit at 2^16) aborts on round-off and is redone
    at a longer length; the residue stays exact."""
    p = 27 * 65536 - 5
    while any(p % d == 0 for d in (3, 5, 7, 11, 13)):
        p -= 2
    k = 40
    r = gpu.run(p, iters=k, n=65536, want_words=True)
    assert r["status"] == 0 and r["escalations"] >= 1 and r["n"] > 65536
    assert r["words"] == oracle.ll_gmp(p, k)[2]


# ---- the two-pass Goldilocks NTT engine (exact: no round-off) ---------------------------------

def _odd_candidate(p):
    p |= 1
    while any(p % d == 0 for d in (3, 5, 7, 11, 13)):
        p -= 2
    return p


@pytest.mark.parametrize("logn", range(14, 24))
def test_ntt_every_large_length_full_residue(gpu, oracle, logn):
    """Every two-pass NTT length at its exactness bound ceil(p/N) = (63 - log2 N)/2 (the widest
    digits the 64-bit field holds), full residue past the first wrap-around."""
    n = 1 << logn
    p = _odd_candidate(((63 - logn) // 2) * n - 1)
    k = p.bit_length() + 4
    r = gpu.run(p, iters=k, n=n, engine="ntt", want_words=True)
    assert r["status"] == 0 and r["n"] == n and r["iters"] == k
    assert r["words"] == oracle.ll_gmp(p, k)[2]
    assert r["max_err"] == 0.0


@pytest.mark.parametrize("logn", [14, 17, 20])
def test_ntt_large_length_low_digit_floor(gpu, oracle, logn):
    """The NTT's lowest usable bits per digit (4 floor(p/N) >= log2 N + 12), where the carry
    chain is longest relative to the digit size."""
    n = 1 << logn
    b = -(-(logn + 12) // 4)
    p = _odd_candidate(b * n + n // 3)
    k = p.bit_length() + 4
    r = gpu.run(p, iters=k, n=n, engine="ntt", want_words=True)
    assert r["status"] == 0 and r["n"] == n
    assert r["words"] == oracle.ll_gmp(p, k)[2]


@pytest.mark.parametrize("p,k", [(1257787, 240), (1257787, 1000), (1257787, 10000)])
def test_ntt_config_p1257787(gpu, p, k):
    """p = 1,257,787 on the NTT at its own length (2^16): res64 vs the reference GMP engine."""
    r = gpu.run(p, iters=k, engine="ntt")
    assert r["status"] == 0 and r["n"] == 65536
    assert r["res64"] == _after()[(p, k)]


def test_ntt_config_sweep_primes_1000(gpu):
    g = load_json("appendix.json")
    after = _after()
    for p in g["sweep_primes"]:
        r = gpu.run(p, iters=1000, engine="ntt")
        assert r["status"] == 0 and r["n"] in (1 << 20, 1 << 21), p
        assert r["res64"] == after[(p, 1000)], p


@pytest.mark.parametrize("k", [34, 1000])
def test_ntt_config_largest_p136279841(gpu, k):
    r = gpu.run(136279841, iters=k, engine="ntt")
    assert r["status"] == 0 and r["n"] == 1 << 23
    assert r["res64"] == _after()[(136279841, k)]


def test_ntt_test_object_pieces(gpu):
    """llg_test_* on the NTT engine: iterating in pieces equals one run, and equals the FP64
    engine's residue for the same squarings."""
    p = 3021377
    t = gpu.Test(p, 0, engine="ntt")
    t.start()
    t.iterate(1)
    t.iterate(998)
    mid = t.read()  # start did the first squaring
    assert mid["iters"] == 1000 and mid["res64"] == gpu.run(p, iters=1000, engine="ntt")["res64"]
    t.read()  # two reads in a row
    t.iterate(1000)
    r = t.read(want_words=True)
    assert r["iters"] == 2000 and r["max_err"] == 0.0
    one = gpu.run(p, iters=2000, engine="ntt", want_words=True)
    f = gpu.run(p, iters=2000, n=1 << 18, want_words=True)
    assert r["words"] == one["words"] == f["words"]
    with pytest.raises(gpu.LlgError):
        t.errlog(10)
    t.close()


def test_ntt_readme_interim_residue(gpu):
    r = gpu.run(3021377, iters=20000, engine="ntt")
    assert r["res64"] == 0xCE811E3772129824


@pytest.mark.parametrize("engine", ["fp64", "ntt"])
def test_config_p1257787_full_run_trace(gpu, engine):
    """p = 1,257,787 (a Mersenne exponent) at N = 65536, all 1,257,785 squarings: res64 every 10^4
    squarings equals the GMP trace (tests/golden/trace_1257787.json), the final residue is zero, and
    (FP64) the worst round-off over the run, and of every logged squaring, stays <= 0.4."""
    tr = load_json("trace_1257787.json")
    p, every = tr["p"], tr["every"]
    t = gpu.Test(p, 65536, engine)
    t.start()
    done = 1
    for i, want in enumerate(tr["res64"]):
        k = every * (i + 1)
        t.iterate(k - done)
        done = k
        r = t.read()
        assert r["iters"] == k and r["res64"] == int(want, 16), (engine, k)
    t.iterate(p - 2 - done)
    r = t.read()
    assert r["iters"] == p - 2 and r["is_zero"] and r["res64"] == 0
    assert r["status"] == 0 and r["max_err"] <= 0.4
    if engine == "fp64":
        log = t.errlog(65536)
        assert len(log) == 65536 and 0.0 < max(log) <= r["max_err"] + 1e-7
    t.close()


@pytest.mark.parametrize("logn", [18, 20, 21, 22, 23])
def test_every_split_full_residue(gpu, oracle, logn):
    """Every row x column split the two-pass FP64 kernels implement at this length (the
    autotuner's choices) gives the exact residue."""
    n = 1 << logn
    p = _odd_candidate(int(16.5 * n))
    k = p.bit_length() + 4
    want = oracle.ll_gmp(p, k)[2]
    splits = gpu.large_splits(logn)
    assert len(splits) >= 1
    try:
        for c in splits:
            gpu.set_large_split(logn, *c)
            assert gpu.get_large_split(logn) == c
            r = gpu.run(p, iters=k, n=n, want_words=True)
            assert r["status"] == 0 and r["words"] == want, (logn, c)
    finally:
        gpu.set_large_split(logn, -1)


def test_splits_p136279841_res64(gpu):
    after = _after()
    try:
        for c in gpu.large_splits(23):
            gpu.set_large_split(23, *c)
            r = gpu.run(136279841, iters=1000, n=1 << 23)
            assert r["res64"] == after[(136279841, 1000)], c
    finally:
        gpu.set_large_split(23, -1)


def test_device_residue_rebuild_matches_host(gpu):
    """llg_residue_from_digits_device against the host rebuild on the same digits: random digits
    of every size class (balanced, wide, tiny), the edge values (zero, 2^p - 1 == 0, -1), one-word
    and large residues, power-of-two and 3 x 2^k lengths."""
    import random
    import torch
    rng = random.Random(5)
    cases = [(61, 4), (127, 32), (4423, 256), (44497, 3072), (330017, 16384), (1257787, 65536),
             (22000007, 1 << 20)]
    for p, n in cases:
        b = -(-p // n)
        for spread in (1 << (b - 1), 1 << min(b + 12, 30), 3):
            d = [rng.randint(-spread, spread) for _ in range(n)]
            dd = torch.tensor(d, dtype=torch.int32, device="cuda")
            got = gpu.residue_from_digits_device(p, n, dd.data_ptr(), want_words=True)
            want = gpu.residue_from_digits(p, n, d)
            assert got == want, (p, n, spread)
            assert gpu.residue_from_digits_device(p, n, dd.data_ptr())[:2] == want[:2]
    p, n = 127, 32
    bits = [-(-((j + 1) * p) // n) - (-(-(j * p) // n)) for j in range(n)]
    for d in ([0] * n, [(1 << x) - 1 for x in bits], [-1] + [0] * (n - 1), [1 << 30] * n, [-(1 << 30)] * n):
        dd = torch.tensor(d, dtype=torch.int32, device="cuda")
        assert gpu.residue_from_digits_device(p, n, dd.data_ptr(), want_words=True) == gpu.residue_from_digits(p, n, d)


# ---- state load, snapshot escalation and the bounded waits --------------------------------------

@pytest.mark.parametrize("engine,n1,n2", [("fp64", 1 << 18, 1 << 18), ("fp64", 1 << 18, 1 << 19),
                                           ("ntt", 1 << 18, 1 << 19), ("fp64", 1 << 19, 1 << 18)])
def test_load_resumes_exactly(gpu, oracle, engine, n1, n2):
    """llg_test_load: a residue read after k squarings at one length, re-digitised on the GPU at
    the same, a longer or a shorter length (or from the other engine), resumes bit-exactly. p is
    usable at both 2^18 and 2^19 (17.2 and 8.6 bits per digit)."""
    p, k, m = _odd_candidate(4500000), 300, 200
    a = gpu.Test(p, n1)
    a.start()
    a.iterate(k - 1)
    w = a.read(want_words=True)["words"]
    a.close()
    b = gpu.Test(p, n2, engine)
    b.load(w, k)
    b.iterate(m - 1)
    r = b.read(want_words=True)
    b.close()
    assert r["iters"] == k + m and r["status"] == 0
    assert r["words"] == oracle.ll_gmp(p, k + m)[2]


def test_corrupted_state_changes_res64(gpu):
    """The exit-3 contract of the reference driver (PerfNumMultiCLL.py:123-129, 234) rests on a
    wrong residue showing in res64: one flipped bit of an interim state, loaded and run on, ends at
    a res64 different from the reference's; the unflipped state ends at the reference's."""
    p, k, total = 1257787, 5000, 10000
    want = int(load_json("trace_1257787.json")["res64"][0], 16)  # after 10^4 squarings
    a = gpu.Test(p, 65536)
    a.start()
    a.iterate(k - 1)
    w = a.read(want_words=True)["words"]
    a.close()
    for flip in (None, (1000, 17), (0, 0)):
        words = list(w)
        if flip:
            words[flip[0]] ^= 1 << flip[1]
        t = gpu.Test(p, 65536)
        t.load(words, k)
        t.iterate(total - k - 1)
        r = t.read()
        t.close()
        assert r["iters"] == total
        assert (r["res64"] == want) == (flip is None), flip


def _later_chunk_exceeding(log, chunk):
    """First chunk c >= 2 of the per-squaring round-off log whose worst value exceeds every earlier
    chunk's, with the bound halfway between the two; None when the first chunk holds the maximum."""
    run = max(log[1:chunk + 1])
    for c in range(2, (len(log) - 1) // chunk + 1):
        m = max(log[(c - 1) * chunk + 1:c * chunk + 1])
        if m > run:
            return c, (run + m) / 2
        run = max(run, m)
    return None


def test_escalation_resumes_from_snapshot(gpu):
    """A round-off abort in the middle of a two-pass run is redone from the last checkpoint at the
    next length: escalations == 1 and the residue equals the exact NTT engine's. The round-off bound
    is set between the worst round-off of the chunks of 4096 squarings before some chunk j >= 2 and
    chunk j's own (read from the run's per-squaring log), so the checks before j pass and check j
    fails; the engine's arithmetic is deterministic, so the run under llg_run sees the same
    round-off. Exponents at ~19 bits per digit are tried until one's log has such a chunk."""
    n, chunk, total = 65536, 4096, 60000
    for p in (1257787, 1250003, 1245011, 1253513, 1239017, 1247509):
        t = gpu.Test(p, n)
        t.start()
        t.iterate(total - 1)
        log = t.errlog(total)  # log[e]: worst round-off of squaring e (e >= 1)
        t.close()
        found = _later_chunk_exceeding(log, chunk)
        if found:
            break
    assert found, "no exponent had a later chunk above its earlier ones"
    j, limit = found
    k = j * chunk + 1000  # past the abort, inside the redone chunk's successor
    old = gpu.get_roundoff_limit()
    try:
        gpu.set_roundoff_limit(limit)
        r = gpu.run(p, iters=k, n=n, want_words=True)
    finally:
        gpu.set_roundoff_limit(old)
    assert r["status"] == 0 and r["escalations"] == 1 and r["n"] > n, (p, r["n"], j, limit)
    want = gpu.run(p, iters=k, engine="ntt", want_words=True)
    assert r["words"] == want["words"]


def test_withheld_wrap_times_out_and_engine_recovers(gpu, oracle):
    """The failure path of the bounded device-side waits: one row pass whose wrap-around job is
    withheld (its flag can never arrive) and whose waits give up after 1000 sleeps. The kernel
    returns, the call reports LLG_E_TIMEOUT quickly, and a following normal run in the same process
    is bit-exact."""
    import time
    p, n = 1257787, 1 << 16
    t = gpu.Test(p, n)
    t.start()
    t.iterate(9)
    t0 = time.perf_counter()
    with pytest.raises(gpu.LlgError) as e:
        t.diag_withhold_wrap(1000)
    assert e.value.code == 6  # LLG_E_TIMEOUT
    assert time.perf_counter() - t0 < 10.0
    t.close()
    r = gpu.run(p, iters=240, n=n)
    assert r["status"] == 0 and r["res64"] == _after()[(p, 240)]


# ---- the {3, 5} x 2^k two-pass lengths (columns of R0 x 512 complex) ---------------------------

MIXED_LARGE = [r << k for r in (3, 5) for k in range(18, 22)]


@pytest.mark.parametrize("n", MIXED_LARGE)
def test_mixed_large_length_full_residue(gpu, oracle, n):
    """Every two-pass length R0 x 2^k at its fewest usable bits per digit (the longest carry
    chains relative to the digit size, and the cheapest oracle run), full residue past the first
    wrap-around."""
    b = -(-((n - 1).bit_length() + 12) // 4)  # 4 floor(p/N) >= ceil(log2 N) + 12
    p = _odd_candidate(b * n + n // 3)
    k = p.bit_length() + 4
    r = gpu.run(p, iters=k, n=n, want_words=True)
    assert r["status"] == 0 and r["n"] == n and r["iters"] == k
    assert r["words"] == oracle.ll_gmp(p, k)[2]


@pytest.mark.parametrize("n", [3 << 18, 5 << 18, 3 << 19])
def test_mixed_large_length_typical_digits(gpu, oracle, n):
    """The same lengths at ~17 bits per digit, where the round-off is largest, over enough
    squarings for the residue to be random."""
    p = _odd_candidate(17 * n + 12345)
    k = 40
    r = gpu.run(p, iters=k, n=n, want_words=True)
    assert r["status"] == 0 and r["n"] == n and r["escalations"] == 0 and r["max_err"] < 0.4
    assert r["words"] == oracle.ll_gmp(p, k)[2]


def test_sweep_primes_at_their_own_length(gpu):
    """The 8 seeded primes of [20M, 25M] at the engine's default length (<= 18 bits per digit):
    5 x 2^18 or 3 x 2^19 instead of 2^21, no escalation, round-off <= 0.4, res64 after 1000
    squarings equal to the reference GMP engine's."""
    g = load_json("appendix.json")
    after = _after()
    for p in g["sweep_primes"]:
        r = gpu.run(p, iters=1000)
        assert r["status"] == 0 and r["n"] <= 3 << 19 and r["n"] in (5 << 18, 3 << 19), (p, r["n"])
        assert r["escalations"] == 0 and r["max_err"] <= 0.4, (p, r["max_err"])
        assert r["res64"] == after[(p, 1000)], p


def test_mixed_large_load_and_interim(gpu, oracle):
    """llg_test_* at a mixed length: pieces equal one run, a residue loaded from 2^20 resumes at
    5 x 2^18 bit-exactly."""
    p = 20357693
    t = gpu.Test(p, 1 << 21)
    t.start()
    t.iterate(99)
    w = t.read(want_words=True)["words"]
    t.close()
    m = gpu.Test(p, 5 << 18)
    m.load(w, 100)
    m.iterate(49)
    mid = m.read()
    m.iterate(50)
    r = m.read(want_words=True)
    m.close()
    assert mid["iters"] == 150 and r["iters"] == 200 and r["n"] == 5 << 18
    assert r["res64"] == gpu.run(p, iters=200, n=5 << 18)["res64"]
    assert mid["res64"] == gpu.run(p, iters=150, n=1 << 21)["res64"]


def test_repeated_call_reuses_the_kept_test_exactly(gpu):
    """llg_run keeps its last two-pass test for the next call on the same exponent, length and
    split: the repeat uploads no tables and gives the same residues, at other iteration counts too
    (each checked against the reference GMP engine); llg_release_cached frees it, and the next call
    builds a fresh one."""
    gold = {(d["p"], d["k"]): int(d["res64"], 16) for d in load_json("appendix.json")["after"]}
    p, n = 1257787, 1 << 16
    gpu.release_cached()
    h0 = gpu.h2d_bytes()
    a = gpu.run(p, iters=1000, n=n)
    h1 = gpu.h2d_bytes()
    b = gpu.run(p, iters=1000, n=n)
    h2 = gpu.h2d_bytes()
    c = gpu.run(p, iters=10000, n=n)
    d = gpu.run(p, iters=240, n=n)
    for r, k in ((a, 1000), (b, 1000), (c, 10000), (d, 240)):
        assert r["status"] == 0 and r["n"] == n and r["res64"] == gold[(p, k)], (k, r)
    assert h1 - h0 > 10000       # tables of the fresh test (~22 KB at 2^16)
    assert h2 - h1 < 1000        # the kept test: no tables again
    gpu.release_cached()
    h3 = gpu.h2d_bytes()
    e = gpu.run(p, iters=1000, n=n)
    assert gpu.h2d_bytes() - h3 > 10000 and e["res64"] == gold[(p, 1000)]
