"""Oracle parity of the kernel configurations the benchmark's ensemble times.

The 512-particle ensemble (grid sizes 128..512) spends most of its time at
n = 384 and 512, where the autotuner picks the warp-independent row kernels (E8
row A in 64-thread groups and the packed two-row row B at 512, whole-warp E12
rows at 384) and the alternative column plans (E16 at 512, E12 at 384).  These
tests force exactly those families (ESC_ROWS / ESC_COLS) on batches of three
particles per size and compare every particle with the CPU oracle
(core_shell.jl:84-103 restated in oracle/core_shell_oracle.py) over 41 steps,
which crosses one captured 32-step graph chunk:
  * FP64 to 1e-12 relative on c and on every history column;
  * the mixed mode to its stated bound, against the oracle itself.
The single large grids are held to the oracle over 20 steps.
"""
import os

import numpy as np
import pytest

import esc
from oracle import core_shell_oracle as orc

pytestmark = pytest.mark.gpu

STEPS = 41
RTOL_FP64 = 1e-12
# mixed mode after 41 steps: FP32 field arithmetic on an FP64 state (c within
# 1e-6 of max|c|, history columns within 1e-6 of their scale, mass to 1e-12)
RTOL_MIXED = 1e-6


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def hist_rel(h, ho):
    return [float(np.max(np.abs(h[:, j] - ho[:, j])) / max(np.max(np.abs(ho[:, j])), 1e-300)) for j in range(6)]


def ensemble_particles(sizes, seed0):
    """Particles drawn like the benchmark ensemble: R ~ U(0.25, 0.42) n, w = 2, sampled P, chi, kappa."""
    rng = np.random.default_rng(seed0)
    out = []
    for k, n in enumerate(sizes):
        phi = orc.particle_disc(n, 1.0, rng.uniform(0.25, 0.42) * n, 2.0)
        c0 = orc.interior_noise(phi, seed0 + k)
        p = esc.Parameters(P=5.0 * rng.uniform(0.5, 2.0), chi=0.5 * rng.uniform(0.5, 1.5),
                           kappa=2.0 * rng.uniform(0.5, 2.0))
        po = orc.Parameters(A=p.A, B=p.B, chi=p.chi, P=p.P, ca=p.ca, cb=p.cb, cc=p.cc, kappa=p.kappa,
                            mobility=p.mobility, Q=p.Q)
        out.append((n, c0, phi, p, po))
    return out


_ORACLE = {}


def oracle_runs(parts, key):
    if key not in _ORACLE:
        orc.set_workers(os.cpu_count() or 1)
        try:
            _ORACLE[key] = [orc.run_simulation(c0, phi, dt=0.01, steps=STEPS, p=po) for (_, c0, phi, _, po) in parts]
        finally:
            orc.set_workers(1)
    return _ORACLE[key]


PARTS_SEED = 900
SIZES = [384, 512, 384, 512, 384, 512]


@pytest.mark.parametrize("cols", ["alt", "block"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_bench_families_against_oracle(prec, cols, monkeypatch):
    monkeypatch.setenv("ESC_ROWS", "warp")
    monkeypatch.setenv("ESC_COLS", cols)
    parts = ensemble_particles(SIZES, PARTS_SEED)
    with esc.Batch([x[2] for x in parts], params=[x[3] for x in parts], precision=prec) as b:
        cs, hs, bad = b.run([x[1] for x in parts], dt=0.01, steps=STEPS)
        desc = {d["n"]: d for d in b.describe()}
    assert bad == [-1] * len(parts)
    want_cols = {"alt": "block-alt-plan", "block": "block"}[cols]
    for n in (384, 512):
        # the FP64 plan at 384 already is the alternative plan (E12), so it reports "block"
        ok = desc[n]["cols"] == want_cols or (prec == "fp64" and n == 384 and desc[n]["cols"] == "block")
        assert desc[n]["rows"] == "warp" and ok, desc[n]
    tol = RTOL_FP64 if prec == "fp64" else RTOL_MIXED
    for (n, c0, phi, p, po), c, h, (co, ho) in zip(parts, cs, hs, oracle_runs(parts, "ens")):
        assert rel(c, co) < tol, (n, prec, cols, rel(c, co))
        hr = hist_rel(h, ho)
        assert max(hr) < tol, (n, prec, cols, hr)
        assert np.max(np.abs(h[:, 1] - c0.mean())) < 1e-12          # mass, FP64 in both modes


def test_tuner_choice_on_the_ensemble_sizes():
    """Whatever the tuner picks for the five ensemble sizes (two particles each) agrees with the oracle."""
    sizes = [128, 192, 256, 384, 512] * 2
    parts = ensemble_particles(sizes, 950)
    with esc.Batch([x[2] for x in parts], params=[x[3] for x in parts], precision="fp64") as b:
        cs, hs, bad = b.run([x[1] for x in parts], dt=0.01, steps=STEPS)
    assert bad == [-1] * len(parts)
    for (n, c0, phi, p, po), c, h, (co, ho) in zip(parts, cs, hs, oracle_runs(parts, "tuner")):
        assert rel(c, co) < RTOL_FP64, n
        assert max(hist_rel(h, ho)) < RTOL_FP64, n


_LARGE = {}


def large_case(n, steps):
    if (n, steps) not in _LARGE:
        phi = orc.particle_disc(n, 1.0, 0.39 * n, 2.0)
        c0 = orc.whole_field_noise(n, 1)
        orc.set_workers(os.cpu_count() or 1)
        try:
            _LARGE[(n, steps)] = (c0, phi) + orc.run_simulation(c0, phi, dt=0.01, steps=steps)
        finally:
            orc.set_workers(1)
    return _LARGE[(n, steps)]


@pytest.mark.parametrize("n", [1024, 4096])
def test_large_single_grid_20_steps_fp64(n):
    """The single-grid configurations (1024^2 disc, 4096^2) over 20 steps against the oracle."""
    c0, phi, co, ho = large_case(n, 20)
    c, h = esc.run_simulation(c0, phi, dt=0.01, steps=20)
    assert rel(c, co) < RTOL_FP64
    assert max(hist_rel(h, ho)) < RTOL_FP64
