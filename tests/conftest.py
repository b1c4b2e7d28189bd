import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "mersenneprime_python_cpp_gmp_benchmark_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def _have_gpu():
    try:
        from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
        llgpu.device_info()
        return True
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """The ctypes binding of the C-ABI, on a machine with a GPU (skips the test without one)."""
    from mersenneprime_python_cpp_gmp_benchmark_b200 import llgpu
    llgpu.lib()  # a missing library is a failure, not a skip
    if not _have_gpu():
        pytest.skip("no CUDA device")
    return llgpu


@pytest.fixture(scope="session")
def ll(gpu):
    """The product's `lucaslehmer` module (reference surface)."""
    import lucaslehmer
    assert os.path.dirname(os.path.abspath(lucaslehmer.__file__)) == PKG
    return lucaslehmer


@pytest.fixture(scope="session")
def lc(gpu):
    import lucaslehmer_cuda
    assert os.path.dirname(os.path.abspath(lucaslehmer_cuda.__file__)) == PKG
    return lucaslehmer_cuda


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    o.lib()
    return o


def load_json(name):
    import json
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def load_range():
    rows = {}
    with open(os.path.join(GOLDEN, "range_100001.csv")) as f:
        for line in f:
            if line.startswith("#"):
                continue
            p, v, r, h = line.strip().split(",")
            rows[int(p)] = (v == "1", int(r, 16), h)
    return rows


KNOWN = [2, 3, 5, 7, 13, 17, 19, 31, 61, 89, 107, 127, 521, 607, 1279, 2203, 2281, 3217, 4253, 4423]


def known_exponents():
    with open(os.path.join(GOLDEN, "known_mp_list.txt")) as f:
        return sorted(int(x) for x in f.read().split())
