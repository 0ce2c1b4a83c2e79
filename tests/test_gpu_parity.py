"""GPU parity: the CUDA library (through the C ABI) against the CPU oracle.

FP64 mode must match the oracle to 1e-12 relative on c and on every history
column (core_shell.jl:84-103 restated in oracle/core_shell_oracle.py); the mixed
mode is held to its stated error bound.
"""
import numpy as np
import pytest

import esc
from oracle import core_shell_oracle as orc

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def case(n, seed=5749):
    return orc.initial_fields(n, radius=70.0 * n / 256, width=max(1.0, 4.0 * n / 256), seed=seed)


def hist_rel(h, ho):
    # column-wise relative error; time column exact
    out = []
    for j in range(6):
        scale = max(np.max(np.abs(ho[:, j])), 1e-300)
        out.append(float(np.max(np.abs(h[:, j] - ho[:, j])) / scale))
    return out


@pytest.mark.parametrize("n,steps", [(8, 5), (12, 7), (16, 10), (24, 10), (32, 20), (48, 20),
                                     (64, 50), (96, 30), (128, 30), (192, 20)])
def test_fp64_matches_oracle_small(n, steps):
    c0, phi = case(n)
    c, h = esc.run_simulation(c0, phi, dt=0.01, steps=steps)
    co, ho = orc.run_simulation(c0, phi, dt=0.01, steps=steps)
    assert rel(c, co) < RTOL_FP64
    hr = hist_rel(h, ho)
    assert max(hr) < RTOL_FP64, hr


@pytest.mark.parametrize("n,steps", [(256, 20), (384, 5), (512, 5), (1024, 2)])
def test_fp64_matches_oracle_sizes(n, steps):
    c0, phi = case(n)
    c, h = esc.run_simulation(c0, phi, dt=0.01, steps=steps)
    co, ho = orc.run_simulation(c0, phi, dt=0.01, steps=steps)
    assert rel(c, co) < RTOL_FP64
    assert max(hist_rel(h, ho)) < RTOL_FP64


def test_default_example_1000_steps_fp64():
    """The default core_shell.jl example (256^2, dt=0.01, 1000 steps, t=10)."""
    c0, phi = orc.initial_fields(256)
    c, h = esc.run_simulation(c0, phi, dt=0.01, steps=1000)
    orc.set_workers(8)
    co, ho = orc.run_simulation(c0, phi, dt=0.01, steps=1000)
    assert rel(c, co) < RTOL_FP64
    assert max(hist_rel(h, ho)) < RTOL_FP64
    # checks.jl:28-29 pins
    assert np.max(np.abs(h[:, 1] - c0.mean())) < 1e-12
    assert np.max(np.diff(h[:, 2])) < 1e-8


def test_mixed_default_example_error_bound():
    c0, phi = orc.initial_fields(256)
    c64, h64 = esc.run_simulation(c0, phi, dt=0.01, steps=1000)
    c32, h32 = esc.run_simulation(c0, phi, dt=0.01, steps=1000, precision="mixed")
    assert np.max(np.abs(c32 - c64)) < 1e-5
    assert np.max(np.abs(h32[:, 1] - c0.mean())) < 1e-12
