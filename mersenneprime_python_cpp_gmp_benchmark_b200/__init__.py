"""B200 Lucas-Lehmer engine: a drop-in for the lucaslehmer / lucaslehmer_cuda modules of
wadeghcp/MersennePrime_Python_CPP_GMP_BenchMark.

Layout of this package (all built in-tree by ``build()``):
  libllgpu.so              CUDA kernels for sm_100a behind the C-ABI of include/llgpu.h
  lucaslehmer*.so          pybind11 module, the reference's ``lucaslehmer`` surface
  lucaslehmer_cuda*.so     pybind11 module, the reference's ``lucaslehmer_cuda`` surface
  llgpu.py                 ctypes binding of the C-ABI (what tests and the benchmark call)

The reference's driver imports ``lucaslehmer`` as a top-level module; put this directory on
``sys.path`` (``use_as_lucaslehmer()`` does that) or on ``PYTHONPATH``.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libllgpu.so")


def build(quiet: bool = True) -> None:
    """Compile libllgpu.so and the two pybind11 modules in-tree (nvcc, sm_100a)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", PKG_DIR, "-j4", "PYTHON=" + sys.executable], check=True, stdout=out)


def use_as_lucaslehmer():
    """Make ``import lucaslehmer`` / ``import lucaslehmer_cuda`` resolve to this engine."""
    if PKG_DIR not in sys.path:
        sys.path.insert(0, PKG_DIR)
    import lucaslehmer  # noqa: F401
    import lucaslehmer_cuda  # noqa: F401
    return lucaslehmer, lucaslehmer_cuda
