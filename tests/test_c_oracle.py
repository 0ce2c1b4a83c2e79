"""The two CPU oracles pin each other.

oracle/core_shell_oracle.c restates core_shell.jl:17-103 a second time, in C
with its own FFT (recursive decimation in time over the prime factors of n);
oracle/core_shell_oracle.py uses NumPy and pocketfft.  They share no code, so
their agreement to rounding, and the C oracle's agreement with the golden
fixtures the NumPy oracle wrote, rule out an error in either restatement that
the other does not make.
"""
import glob
import os

import numpy as np
import pytest

from oracle import c_oracle as co
from oracle import core_shell_oracle as orc

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
RTOL = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def hist_rel(h, ho):
    return max(float(np.max(np.abs(h[:, j] - ho[:, j])) / max(np.max(np.abs(ho[:, j])), 1e-300)) for j in range(6))


@pytest.mark.parametrize("n", [1, 2, 3, 5, 6, 8, 10, 12, 16, 24, 27, 48, 96, 128])
def test_own_fft_matches_a_direct_dft(n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    j = np.arange(n)
    w = np.exp(-2j * np.pi * np.outer(j, j) / n)        # direct DFT matrix, independent of any FFT
    ref = w @ a @ w                                        # transform along both axes (w is symmetric)
    f = co.fft2(a)
    assert rel(f, ref) < 1e-13
    assert rel(co.fft2(f, inverse=True), a) < 1e-13


@pytest.mark.parametrize("n,steps,over", [
    (8, 6, {}),
    (12, 10, {"P": 6.0, "chi": 0.6}),
    (24, 15, {"kappa": 3.0, "Q": 0.7}),
    (32, 25, {"A": 2.5, "B": 3.5}),
    (48, 20, {"mobility": 1.5}),
    (96, 8, {"ca": 0.45, "cb": 0.05, "cc": 0.95}),
])
def test_c_oracle_matches_numpy_oracle(n, steps, over):
    c0, phi = orc.initial_fields(n, radius=n / 4, width=max(1.0, n / 32), seed=n)
    p = orc.Parameters(**over)
    c1, h1 = co.run_simulation(c0, phi, dt=0.01, steps=steps, p=p)
    c2, h2 = orc.run_simulation(c0, phi, dt=0.01, steps=steps, p=p)
    assert rel(c1, c2) < RTOL
    assert hist_rel(h1, h2) < RTOL


def test_c_oracle_spacing_and_whole_field_noise():
    n = 32
    phi = orc.particle_disc(n, spacing=0.5, radius=5.0, width=1.0)
    c0 = orc.whole_field_noise(n, seed=7)
    c1, h1 = co.run_simulation(c0, phi, dt=0.005, steps=12, spacing=0.5)
    c2, h2 = orc.run_simulation(c0, phi, dt=0.005, steps=12, spacing=0.5)
    assert rel(c1, c2) < RTOL
    assert hist_rel(h1, h2) < RTOL


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "disc*.npz"))))
def test_c_oracle_reproduces_golden_fixtures(path):
    g = np.load(path)
    p = orc.Parameters(*[float(x) for x in g["params"]])
    c, h = co.run_simulation(g["c0"], g["phi"], dt=float(g["dt"]), steps=int(g["steps"]), p=p)
    assert rel(c, g["c"]) < RTOL
    assert hist_rel(h, g["history"]) < RTOL


def test_c_oracle_conserves_mass_and_reports_nonfinite():
    c0, phi = orc.initial_fields(48, radius=12.0, width=2.0, seed=11)
    _, h = co.run_simulation(c0, phi, dt=0.01, steps=30)
    assert np.max(np.abs(h[:, 1] - h[0, 1])) < 1e-14          # mass (checks.jl:28)
    assert np.max(np.diff(h[:, 2])) < 1e-8                    # energy non-increasing (checks.jl:29)
    bad = c0.copy()
    bad[3, 4] = np.nan
    with pytest.raises(orc.NonFiniteError) as err:
        co.run_simulation(bad, phi, dt=0.01, steps=5)
    assert err.value.step == 0
