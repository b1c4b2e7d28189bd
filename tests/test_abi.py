"""The C-ABI boundary without a GPU: the library loads and exports every function include/llgpu.h
declares, the host-side residue rebuild is exact against the oracle, length selection follows the
reference's rules, and the pybind11 modules expose the reference's surface."""
import ctypes
import os
import random

import pytest

from conftest import PKG


def test_library_exports_every_header_function():
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    names = llgpu.header_functions()
    assert len(names) >= 10
    L = llgpu.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert missing == []


def test_status_strings():
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    L = llgpu.lib()
    for code in range(8):
        assert L.llg_status_string(code)
    assert L.llg_status_string(0) == b"ok"


def _random_digits(rng, p, n, spread):
    return [rng.randint(-spread, spread) for _ in range(n)]


def test_residue_rebuild_matches_oracle(oracle):
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    rng = random.Random(11)
    cases = [(61, 4), (127, 32), (521, 32), (4423, 256), (9689, 512), (20011, 1024), (100003, 8192),
             (1257787, 65536)]
    for p, n in cases:
        b = -(-p // n)
        for spread in (1 << (b - 1), 1 << (b + 12), 3):
            d = _random_digits(rng, p, n, spread)
            z1, r1, w1 = llgpu.residue_from_digits(p, n, d)
            z2, r2, w2 = oracle.rebuild(p, n, d)
            assert (z1, r1, w1) == (z2, r2, w2), (p, n, spread)


def test_residue_rebuild_edge_values(oracle):
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    p, n = 127, 32
    zero = [0] * n
    assert llgpu.residue_from_digits(p, n, zero)[0] is True
    # the all-ones pattern 2^p - 1 is zero
    bits = [-(-((j + 1) * p) // n) - (-(-(j * p) // n)) for j in range(n)]
    ones = [(1 << b) - 1 for b in bits]
    z, r, w = llgpu.residue_from_digits(p, n, ones)
    assert z and r == 0
    # -1 is 2^p - 2
    m1 = [-1] + [0] * (n - 1)
    z, r, w = llgpu.residue_from_digits(p, n, m1)
    assert not z and sum(x << (64 * i) for i, x in enumerate(w)) == (1 << p) - 2


def test_fft_length_rules():
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    assert llgpu.fft_length(63) == 0 and llgpu.fft_length(255) == 0  # exact word kernel below 256
    prev = 0

    def kind(n):  # n = m 2^k with m in {1, 3, 5}, as the reference's lengths (lucaslehmer.cpp:244-254)
        while n % 2 == 0:
            n //= 2
        return n
    for p in (256, 300, 521, 4423, 9689, 20011, 44497, 60013, 80021, 100001, 147456):
        n = llgpu.fft_length(p)
        assert n >= prev and kind(n) in (1, 3, 5)
        assert p / n <= 18.0 and p >= 2 * n
        prev = n
    # the non-power-of-two whole-test lengths
    assert llgpu.fft_length(44497) == 3072 and llgpu.fft_length(80021) == 5120
    assert llgpu.fft_length(100001) == 6144 and llgpu.fft_length(150001) == 10240
    assert llgpu.fft_length(200001) == 12288 and llgpu.fft_length(250001) == 16384
    assert llgpu.fft_length(100001, 19.0) == 6144


def test_run_without_gpu_fails_loudly():
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    try:
        llgpu.device_info()
    except llgpu.LlgError as e:
        assert e.code == 2  # LLG_E_NODEV
        with pytest.raises(llgpu.LlgError):
            llgpu.run(4423)
    else:
        pytest.skip("a GPU is present")


def test_failed_calls_copy_nothing_and_release_is_safe():
    """Without a GPU a call fails before any upload (the library's host-to-device count does not
    move), and releasing the kept two-pass test is a harmless no-op."""
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    try:
        llgpu.device_info()
    except llgpu.LlgError:
        h0 = llgpu.h2d_bytes()
        for p, n in ((136279841, 1 << 23), (1257787, 1 << 16), (4423, 0)):
            with pytest.raises(llgpu.LlgError):
                llgpu.run(p, iters=10, n=n)
        assert llgpu.h2d_bytes() == h0
        llgpu.release_cached()
        llgpu.release_cached()
    else:
        pytest.skip("a GPU is present")


def test_pybind_modules_reference_surface():
    import lucaslehmer as ll
    import lucaslehmer_cuda as lc
    assert os.path.dirname(os.path.abspath(ll.__file__)) == PKG
    for name in ("lucas_lehmer", "lucas_lehmer_split", "lucas_lehmer_fft", "lucas_lehmer_res",
                 "lucas_lehmer_split_res", "lucas_lehmer_fft_res", "fft_res64_after", "gmp_res64_after",
                 "fft_info", "fft_backend", "set_fft_bits_per_word", "bench_square", "primes",
                 "mersenne_digits", "mersenne_str", "gmp_version", "LucasLehmer"):
        assert hasattr(ll, name), name
    for name in ("lucas_lehmer_batch", "ntt_length", "max_exponent", "device_info"):
        assert hasattr(lc, name), name
    # reference tests/test_lucaslehmer.py:5-9,18-19,21-23 (host-only parts)
    assert len(ll.primes(2, 10001)) == 1229
    assert ll.primes(0, 1) == [] and ll.primes(2, 2) == [2] and ll.primes(10, 20) == [11, 13, 17, 19]
    assert ll.mersenne_digits(127) == 39 and ll.mersenne_str(7) == "127"
    assert ll.mersenne_str(127) == str(2**127 - 1)
    c = ll.LucasLehmer()
    out = []
    assert c.sa_getListOfPrimes(out, 2, 10) is True and out == [2, 3, 5, 7]


def test_mersenne_digits_formula_matches_string():
    import sys
    import lucaslehmer as ll
    sys.set_int_max_str_digits(0)
    for p in (3999, 4000, 4001, 4253, 9689, 21701, 44497, 86243):
        assert ll.mersenne_digits(p) == len(str(2**p - 1)), p


def test_tune_file_round_trip(tmp_path, monkeypatch):
    """The autotuner's file format: lines for other devices and lengths are kept, this device's
    lengths are replaced (host-side logic only; the timing itself needs a GPU)."""
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    path = tmp_path / "tune.txt"
    path.write_text("large_split\tOther GPU\t23\t11\t2\nlarge_split\tNVIDIA B200\t22\t9\t4\n")
    monkeypatch.setenv("LLG_TUNE_CACHE", str(path))
    assert llgpu.tune_cache_path() == str(path)
    monkeypatch.setattr(llgpu, "device_info", lambda: ("NVIDIA B200", 148, 0))
    monkeypatch.setattr(llgpu, "large_splits", lambda ln: [(10, 4), (10, 2), (11, 2)])
    monkeypatch.setattr(llgpu, "set_large_split", lambda ln, c, g=0: None)

    class FakeTest:
        def __init__(self, p, n, engine="fp64"):
            self.n = n
        def start(self): pass
        def iterate(self, k): pass
        def time_passes(self, k):
            return (100.0, 90.0)
        def close(self): pass
    monkeypatch.setattr(llgpu, "Test", FakeTest)
    out = llgpu.autotune([22, 23], iters=4, warmup=1)
    assert set(out) == {22, 23} and out[23][0] in ((10, 4), (10, 2), (11, 2))
    lines = path.read_text().splitlines()
    assert "large_split\tOther GPU\t23\t11\t2" in lines
    assert sum(1 for l in lines if l.startswith("large_split\tNVIDIA B200\t22\t")) == 1
    assert sum(1 for l in lines if l.startswith("large_split\tNVIDIA B200\t23\t")) == 1


def test_length_choice_rule():
    """llg_set_length_choice: exponents whose bits-per-digit length is n_rule move to n_use where
    it is usable for them; clearing restores the rule; lengths shorter than the rule's, and
    non-lengths, are refused."""
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    p = 85009  # 16.6 bits per digit at N = 5120, the rule's length
    assert llgpu.fft_length(p) == 5120
    try:
        llgpu.set_length_choice(5120, 8192)
        assert llgpu.get_length_choice(5120) == 8192
        assert llgpu.fft_length(p) == 8192 and llgpu.fft_length(p, 17.0) == 8192
        with pytest.raises(llgpu.LlgError):
            llgpu.set_length_choice(5120, 4096)  # shorter than the rule's length
        with pytest.raises(llgpu.LlgError):
            llgpu.set_length_choice(5000, 8192)  # not a length
    finally:
        llgpu.set_length_choice(5120, 0)
    assert llgpu.fft_length(p) == 5120 and llgpu.get_length_choice(5120) == 5120
