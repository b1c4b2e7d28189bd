"""The reference's driver, PerfNumMultiCLL.py, run unchanged against this engine's modules.

oracle/_ref/driver/ holds the driver and its known_mp_list.txt, copied byte for byte from the
reference by `make -C oracle ref` (build() does it where the reference's sources are present).
Each case runs the script as a subprocess with PYTHONPATH set to the package directory, so its
`import lucaslehmer` / `import lucaslehmer_cuda` load this engine. Checked, as the driver itself
reports them (PerfNumMultiCLL.py:219-235): exit status 0, the hit set equal to known_mp_list.txt
within the range, the --verify pass reporting no mismatch (exit 3 otherwise, :123-129, :234),
and every row's res64 equal to the reference GMP engine's (tests/golden/range_100001.csv).
"""
import json
import os
import subprocess
import sys

import pytest

from conftest import PKG, ROOT, known_exponents, load_range

pytestmark = pytest.mark.gpu

DRIVER_DIR = os.path.join(ROOT, "oracle", "_ref", "driver")
DRIVER = os.path.join(DRIVER_DIR, "PerfNumMultiCLL.py")


@pytest.fixture(scope="module")
def driver(gpu):
    if not os.path.exists(DRIVER):
        pytest.skip("oracle/_ref/driver not built (needs the reference's sources at build time)")

    def run(args, timeout=900):
        env = dict(os.environ, PYTHONPATH=PKG + os.pathsep + os.environ.get("PYTHONPATH", ""))
        return subprocess.run([sys.executable, DRIVER, *args], capture_output=True, text=True,
                              timeout=timeout, env=env, cwd=DRIVER_DIR)

    return run


def _check_rows(out_json, hi):
    with open(out_json) as f:
        doc = json.load(f)
    gold = load_range()
    rows = {row["p"]: row for row in doc["rows"]}
    ps = sorted(rows)
    assert ps == [p for p in sorted(gold) if p <= hi]
    bad = [p for p in ps if int(rows[p]["res64"], 16) != gold[p][1] or rows[p]["mersenne"] != gold[p][0]]
    assert not bad, f"res64 / verdict differs from the reference GMP engine at {bad[:10]}"
    assert doc["hits"] == [p for p in known_exponents() if p <= hi]
    return doc


def _modules_are_ours(proc):
    # the driver prints the `gmp_version` of the module it imported; this engine's says so
    assert "gmp none (b200 engine)" in proc.stdout, proc.stdout[-2000:] + proc.stderr[-2000:]


def test_driver_fft_engine(driver, tmp_path):
    """--engine fft: the default per-exponent path, lucas_lehmer_fft_res from a 16-thread pool."""
    out = tmp_path / "fft.json"
    r = driver(["-t", "16", "-r", "10001", "--engine", "fft", "--json", str(out), "--progress", "0"])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    _modules_are_ours(r)
    doc = _check_rows(out, 10001)
    assert doc["engine"] == "fft" and doc["fft_backend"] == "b200-fp64-ibdwt"


def test_driver_cuda_engine_and_verify(driver, tmp_path):
    """--engine cuda over every prime p <= 100001 (chunks of 2048 per transform length), then a
    second pass with --verify against the first pass's JSON."""
    first = tmp_path / "cuda.json"
    r = driver(["-r", "100001", "--engine", "cuda", "--json", str(first), "--progress", "0"])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    _modules_are_ours(r)
    _check_rows(first, 100001)
    second = tmp_path / "cuda2.json"
    v = driver(["-r", "100001", "--engine", "cuda", "--json", str(second), "--verify", str(first),
                "--progress", "0"])
    assert v.returncode == 0, v.stdout[-2000:] + v.stderr[-2000:]
    assert "9592 checked, 0 mismatches" in v.stderr, v.stderr[-2000:]
    _check_rows(second, 100001)


def test_driver_loop_mode(driver, tmp_path):
    """--loop 2 (torture-test mode): pass 1 is the res64 reference, pass 2 is checked against it."""
    r = driver(["-t", "8", "-r", "3000", "--engine", "fft", "--loop", "2", "--json", str(tmp_path / "loop.json"),
                "--progress", "0"])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "=== pass 2 (verifying against" in r.stderr and "0 mismatches" in r.stderr, r.stderr[-2000:]
    _check_rows(tmp_path / "loop.json", 3000)


def test_driver_gmp_engine_and_list(driver, tmp_path):
    """--engine gmp (the exact engine) on an explicit list, and the prime-count mode. The list spans
    no known exponent it leaves out (the driver exits 2 when one inside [min, max] is not found)."""
    out = tmp_path / "gmp.json"
    r = driver(["-t", "4", "-l", "4423", "4643", "5003", "9689", "9941", "--engine", "gmp", "--json", str(out),
                "--progress", "0"])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    _modules_are_ours(r)
    with open(out) as f:
        doc = json.load(f)
    gold = load_range()
    assert doc["hits"] == [4423, 9689, 9941]
    assert all(int(row["res64"], 16) == gold[row["p"]][1] for row in doc["rows"])
    n = driver(["-n", "2", "100001"])
    assert n.returncode == 0 and "primes in [2, 100001]: 9592" in n.stdout, n.stdout
