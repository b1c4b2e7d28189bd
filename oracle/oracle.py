"""ctypes front end of THE ORACLE (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference arm may import this
module, and only as the checker or the timed CPU side: the product package never imports it.

Functions mirror llref.h; each restates a piece of the reference (file:line given there):
GMP engine (lucaslehmer.cpp:29-58), residue rebuild (lucaslehmer.cpp:312-323), FP64 IBDWT engine
(lucaslehmer.cpp:244-335) and the Goldilocks NTT engine (cuda/ll_ntt.cu:38-195).
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and, when the reference sources are present, oracle/_ref)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "PYTHON=" + sys.executable, "all"], check=True, stdout=out)
    ref = os.environ.get("LL_REFERENCE_SRC", "/root/reference")
    if os.path.exists(os.path.join(ref, "lucaslehmer.cpp")):
        subprocess.run(["make", "-C", HERE, "PYTHON=" + sys.executable, "REF=" + ref, "ref"],
                       check=True, stdout=out)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u64, i64, sz, dbl = ctypes.c_uint64, ctypes.c_int64, ctypes.c_size_t, ctypes.c_double
        P = ctypes.POINTER
        L.orc_ll_gmp.argtypes = [u64, u64, P(u64), P(u64), sz]
        L.orc_ll_gmp.restype = ctypes.c_int
        L.orc_ll_gmp_trace.argtypes = [u64, u64, u64, P(u64), sz]
        L.orc_ll_gmp_trace.restype = ctypes.c_int
        L.orc_rebuild.argtypes = [u64, u64, P(i64), P(u64), P(u64), sz]
        L.orc_rebuild.restype = ctypes.c_int
        L.orc_fft_length.argtypes = [u64, dbl]
        L.orc_fft_length.restype = u64
        L.orc_ibdwt.argtypes = [u64, u64, u64, dbl, P(dbl), P(i64), P(u64), P(u64), sz]
        L.orc_ibdwt.restype = ctypes.c_int
        for name in ("orc_gl_add", "orc_gl_sub", "orc_gl_mul", "orc_gl_pow"):
            getattr(L, name).argtypes = [u64, u64]
            getattr(L, name).restype = u64
        L.orc_ntt_max_bits.argtypes = [u64]
        L.orc_ntt_max_bits.restype = ctypes.c_int
        L.orc_ntt_length.argtypes = [u64]
        L.orc_ntt_length.restype = u64
        L.orc_ntt_tables.argtypes = [u64, P(u64), P(u64), P(u64)]
        L.orc_ntt_tables.restype = ctypes.c_int
        L.orc_ntt.argtypes = [u64, u64, u64, P(i64), P(u64), P(u64), sz]
        L.orc_ntt.restype = ctypes.c_int
        _lib = L
    return _lib


def nwords(p: int) -> int:
    return max(1, (p + 63) // 64)


def words_to_int(words) -> int:
    v = 0
    for i, w in enumerate(words):
        v |= int(w) << (64 * i)
    return v


def residue_hash(words) -> str:
    """64-bit fingerprint of a full residue: blake2b-64 over its little-endian 64-bit words."""
    b = b"".join(int(w).to_bytes(8, "little") for w in words)
    return hashlib.blake2b(b, digest_size=8).hexdigest()


def ll_gmp(p: int, iters: int = 0):
    """(is_zero, res64, words) of s_iters (iters=0: the full p-2) -- lucaslehmer.cpp:29-58."""
    n = nwords(p)
    words = (ctypes.c_uint64 * n)()
    r = ctypes.c_uint64()
    v = lib().orc_ll_gmp(p, iters, ctypes.byref(r), words, n)
    return bool(v), r.value, list(words)


def ll_gmp_trace(p: int, iters: int, every: int):
    n = iters // every
    out = (ctypes.c_uint64 * n)()
    k = lib().orc_ll_gmp_trace(p, iters, every, out, n)
    return list(out)[:max(k, 0)]


def rebuild(p: int, N: int, digits):
    n = nwords(p)
    words = (ctypes.c_uint64 * n)()
    r = ctypes.c_uint64()
    d = (ctypes.c_int64 * N)(*[int(x) for x in digits])
    v = lib().orc_rebuild(p, N, d, ctypes.byref(r), words, n)
    return bool(v), r.value, list(words)


def fft_length(p: int, max_bpw: float = 18.0) -> int:
    return int(lib().orc_fft_length(p, max_bpw))


def ibdwt(p: int, N: int = 0, iters: int = 0, abort_err: float = 0.35, want_digits=False):
    """(verdict, res64, maxerr, words, digits) of the FP64 IBDWT restatement (lucaslehmer.cpp:257-329)."""
    if N == 0:
        N = fft_length(p)
    n = nwords(p)
    words = (ctypes.c_uint64 * n)()
    digits = (ctypes.c_int64 * N)() if want_digits else None
    r = ctypes.c_uint64()
    e = ctypes.c_double()
    v = lib().orc_ibdwt(p, N, iters, abort_err, ctypes.byref(e), digits, ctypes.byref(r), words, n)
    return v, r.value, e.value, list(words), (list(digits) if digits is not None else None)


def ntt(p: int, N: int = 0, iters: int = 0, want_digits=False):
    """(verdict, res64, words, digits) of the Goldilocks NTT restatement (cuda/ll_ntt.cu:74-167)."""
    if N == 0:
        N = int(lib().orc_ntt_length(p))
    n = nwords(p)
    words = (ctypes.c_uint64 * n)()
    digits = (ctypes.c_int64 * N)() if want_digits else None
    r = ctypes.c_uint64()
    v = lib().orc_ntt(p, N, iters, digits, ctypes.byref(r), words, n)
    return v, r.value, list(words), (list(digits) if digits is not None else None)


def ntt_tables(N: int):
    o, r2, inv = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    rc = lib().orc_ntt_tables(N, ctypes.byref(o), ctypes.byref(r2), ctypes.byref(inv))
    if rc != 0:
        raise ValueError(f"no NTT tables for N={N}")
    return o.value, r2.value, inv.value


def primes(lo: int, hi: int):
    """Sieve of Eratosthenes over [lo, hi] (the checker's own; lucaslehmer.cpp:72-80)."""
    if hi < 2:
        return []
    comp = bytearray(hi + 1)
    i = 2
    while i * i <= hi:
        if not comp[i]:
            comp[i * i::i] = b"\x01" * len(range(i * i, hi + 1, i))
        i += 1
    return [i for i in range(max(lo, 2), hi + 1) if not comp[i]]


_ref_mod = None


def reference_module():
    """The reference's own lucaslehmer module, compiled unchanged into oracle/_ref, or None.

    Loaded under the private name ``_oracle_ref.lucaslehmer`` so that it never shadows the
    product's ``lucaslehmer`` module in ``sys.modules``."""
    global _ref_mod
    if _ref_mod is not None:
        return _ref_mod
    import importlib.machinery
    import importlib.util
    import sysconfig
    path = os.path.join(HERE, "_ref", "lucaslehmer" + sysconfig.get_config_var("EXT_SUFFIX"))
    if not os.path.exists(path):
        return None
    loader = importlib.machinery.ExtensionFileLoader("_oracle_ref.lucaslehmer", path)
    spec = importlib.util.spec_from_file_location("_oracle_ref.lucaslehmer", path, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    _ref_mod = mod
    return mod
