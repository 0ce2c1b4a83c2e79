"""Grid sizes without a tuned kernel set, through the runtime-size kernels.

The reference takes any n: make_grid zeroes the derivative Nyquist only when n
is even (core_shell.jl:20), and FFTW transforms every length.  The tuned kernel
sets cover the even 2^a 3^b sizes; every other n from 2 to 4096 (prime factors
up to 127, or any n up to 512) runs on the runtime-size kernels
(csrc/esc_generic.cu).  These tests hold them to the CPU oracle
(core_shell.jl:84-103 restated in oracle/core_shell_oracle.py) at 1e-12 in FP64,
at odd, even, prime and radix-5/7 sizes; force them (ESC_GENERIC=1) at tuned
sizes so that both kernel families meet the same oracle; and check the mixed
precision, batches that mix both families, and the non-finite path.
"""
import os

import numpy as np
import pytest

import esc
from oracle import core_shell_oracle as orc

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def hist_rel(h, ho):
    return max(float(np.max(np.abs(h[:, j] - ho[:, j])) / max(np.max(np.abs(ho[:, j])), 1e-300)) for j in range(6))


def case(n, seed=11):
    return orc.initial_fields(n, radius=0.3 * n, width=max(1.0, n / 64), seed=seed)


def oracle(c0, phi, steps, p=orc.Parameters(), dt=0.01):
    orc.set_workers(os.cpu_count() or 1)
    try:
        return orc.run_simulation(c0, phi, dt=dt, steps=steps, p=p)
    finally:
        orc.set_workers(1)


@pytest.mark.parametrize("n,steps", [(2, 5), (3, 5), (7, 9), (10, 20), (15, 20), (21, 12), (45, 10), (97, 10),
                                     (100, 20), (160, 12), (250, 8), (320, 8), (1000, 5)])
def test_fp64_generic_sizes_match_oracle(n, steps):
    assert esc.supported_size(n)
    c0, phi = case(n)
    c, h = esc.run_simulation(c0, phi, dt=0.01, steps=steps)
    co, ho = oracle(c0, phi, steps)
    assert rel(c, co) < RTOL_FP64, (n, rel(c, co))
    assert hist_rel(h, ho) < RTOL_FP64, (n, hist_rel(h, ho))


@pytest.mark.parametrize("n", [8, 64, 256])
def test_forced_generic_kernels_at_tuned_sizes(n, monkeypatch):
    """ESC_GENERIC=1 runs the runtime-size kernels where a tuned set exists: both families meet the oracle."""
    monkeypatch.setenv("ESC_GENERIC", "1")
    c0, phi = case(n, seed=5)
    c, h = esc.run_simulation(c0, phi, dt=0.01, steps=33)
    co, ho = oracle(c0, phi, 33)
    assert rel(c, co) < RTOL_FP64 and hist_rel(h, ho) < RTOL_FP64


@pytest.mark.parametrize("n", [15, 99, 100])
def test_mixed_generic_within_bound_of_fp64(n):
    c0, phi = case(n, seed=7)
    c64, h64 = esc.run_simulation(c0, phi, dt=0.01, steps=60)
    c32, h32 = esc.run_simulation(c0, phi, dt=0.01, steps=60, precision="mixed")
    assert rel(c32, c64) < 1e-5
    assert np.max(np.abs(h32[:, 1] - h32[0, 1])) < 1e-12          # FP64 state and mass fix
    assert np.max(np.abs(h32[:, 2] - h64[:, 2])) / np.max(np.abs(h64[:, 2])) < 1e-5


def test_batch_mixing_tuned_and_generic_sizes():
    sizes = [15, 64, 100, 48, 15, 81]
    parts = [case(n, seed=20 + k) for k, n in enumerate(sizes)]
    steps = 34                                                   # crosses a captured 32-step chunk
    with esc.Batch([x[1] for x in parts], precision="fp64") as b:
        cs, hs, bad = b.run([x[0] for x in parts], dt=0.01, steps=steps)
    assert bad == [-1] * len(parts)
    for n, (c0, phi), c, h in zip(sizes, parts, cs, hs):
        co, ho = oracle(c0, phi, steps)
        assert rel(c, co) < RTOL_FP64, n
        assert hist_rel(h, ho) < RTOL_FP64, n


def test_generic_long_run_properties():
    """checks.jl:19-20 at an odd size: mass drift < 1e-12 and energy non-increasing over 1000 steps."""
    c0, phi = case(75, seed=9)
    c, h = esc.run_simulation(c0, phi, dt=0.01, steps=1000)
    assert np.max(np.abs(h[:, 1] - c0.mean())) < 1e-12
    assert np.max(np.diff(h[:, 2])) < 1e-8


def test_generic_nonfinite_reports_step_and_keeps_c():
    c0, phi = case(21)
    bad = c0.copy()
    bad[4, 9] = np.inf
    with pytest.raises(esc.NonFiniteError) as ei:
        esc.run_simulation(bad, phi, dt=0.01, steps=4)
    assert ei.value.step == 0


_CACHED_CHILD = r"""
import sys
import numpy as np
import esc
from oracle import core_shell_oracle as orc
n = int(sys.argv[1])
c0, phi = orc.initial_fields(n, radius=0.3 * n, width=max(1.0, n / 64), seed=5)
c, h = esc.run_simulation(c0, phi, dt=0.01, steps=9)
np.savez(sys.argv[2], c=c, h=h, c0=c0, phi=phi)
"""


@pytest.mark.parametrize("n", [128, 256])
def test_forced_generic_ignores_cached_tuned_decisions(n, tmp_path):
    """A decision the tuner kept for the tuned kernel set of the same (n, precision,
    instance count) -- here the alternative column plan with warp rows, as a tuner
    cache file holds it -- does not apply to the runtime-size kernels, which have
    one family each.  Fresh process: the cache file is read once per process."""
    import subprocess
    import sys
    cache = tmp_path / "tune.jsonl"
    cache.write_text("".join(f'{{"n": {n}, "prec": {p}, "count": 1, "rows": 2, "cols": 2}}\n' for p in (0, 1)))
    out = tmp_path / "run.npz"
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, ESC_TUNE_CACHE=str(cache), ESC_GENERIC="1",
               PYTHONPATH=os.pathsep.join([root, os.path.join(root, "embedded-spinodal-core-shell-julia_b200"),
                                           os.environ.get("PYTHONPATH", "")]))
    r = subprocess.run([sys.executable, "-c", _CACHED_CHILD, str(n), str(out)], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    d = np.load(out)
    co, ho = oracle(d["c0"], d["phi"], 9)
    assert rel(d["c"], co) < RTOL_FP64 and hist_rel(d["h"], ho) < RTOL_FP64
