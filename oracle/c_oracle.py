"""ctypes front end of the second CPU oracle (oracle/core_shell_oracle.c).

TEST INFRASTRUCTURE ONLY.  The tests, the smoke check and the CPU-baseline leg
of the benchmark may use it; the product path (the CUDA library and its Python
binding) never does.

The C oracle restates core_shell.jl:17-103 with its own FFT, independently of
the NumPy oracle (core_shell_oracle.py): the two agreeing to rounding pins both.
`build()` compiles it with gcc into oracle/libcsoracle.so (plain IEEE FP64: no
fast-math, no FMA contraction).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from . import core_shell_oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCE = os.path.join(HERE, "core_shell_oracle.c")
LIBRARY = os.path.join(HERE, "libcsoracle.so")

_lib = None


def build(force: bool = False) -> str:
    """Compile the C oracle if it is missing or older than its source; returns the path."""
    if force or not os.path.exists(LIBRARY) or os.path.getmtime(LIBRARY) < os.path.getmtime(SOURCE):
        subprocess.run(["gcc", "-O2", "-std=c99", "-ffp-contract=off", "-fPIC", "-shared", "-o", LIBRARY, SOURCE,
                        "-lm"], check=True)
    return LIBRARY


def _load():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.cso_run_simulation.restype = ctypes.c_int
        _lib.cso_run_simulation.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp, dp, ctypes.c_int, ctypes.c_double,
                                            dp, dp, ctypes.POINTER(ctypes.c_int64)]
        _lib.cso_fft2.restype = ctypes.c_int
        _lib.cso_fft2.argtypes = [ctypes.c_int, dp, ctypes.c_int]
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def run_simulation(c0, phi, dt: float = 0.01, steps: int = 1000, spacing: float = 1.0,
                   p: orc.Parameters = orc.Parameters()):
    """Same contract as core_shell_oracle.run_simulation: returns (c, history (steps+1, 6));
    a non-finite field raises core_shell_oracle.NonFiniteError after its row is recorded."""
    lib = _load()
    c0 = np.ascontiguousarray(c0, dtype=np.float64)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    n = c0.shape[0]
    if c0.shape != (n, n) or phi.shape != (n, n):
        raise ValueError("c0 and phi must be square and of one size")
    params = np.array(p.as_tuple(), dtype=np.float64)
    c = np.empty_like(c0)
    hist = np.zeros((6, steps + 1))  # column-major (steps+1) x 6, as the Julia matrix
    bad = ctypes.c_int64(-1)
    st = lib.cso_run_simulation(n, float(spacing), _dp(phi), _dp(params), _dp(c0), int(steps), float(dt), _dp(c),
                                _dp(hist), ctypes.byref(bad))
    if st == 3:
        raise orc.NonFiniteError(int(bad.value))
    if st != 0:
        raise RuntimeError(f"C oracle failed with status {st}")
    return c, hist.T.copy()


def fft2(a: np.ndarray, inverse: bool = False) -> np.ndarray:
    """The C oracle's own 2-D transform (unnormalised forward, 1/n^2 inverse)."""
    lib = _load()
    z = np.ascontiguousarray(a, dtype=np.complex128).copy()
    n = z.shape[0]
    if z.shape != (n, n):
        raise ValueError("square field expected")
    st = lib.cso_fft2(n, _dp(z.view(np.float64)), 1 if inverse else 0)
    if st != 0:
        raise RuntimeError(f"C oracle FFT failed with status {st}")
    return z
