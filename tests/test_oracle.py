"""The CPU oracle pinned against the reference's own checks and known answers.

The reference's test file checks.jl (30 lines) asserts physics identities and
run properties; check-results.txt records one run of it.  The noise of the
reference comes from Julia's MersenneTwister, which cannot be reproduced
without Julia, so realisation-dependent numbers become bands calibrated across
seeds; realisation-independent identities are pinned exactly as checks.jl does.
"""
import os

import numpy as np
import pytest

from oracle import core_shell_oracle as orc

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
P = orc.Parameters()


def setup64():
    c, phi = orc.initial_fields(64, radius=16.0)          # checks.jl:4
    return c, phi, orc.make_grid(64, 1.0), orc.geometry(phi, P)


def test_parameters_defaults():
    # core_shell.jl:4-15
    assert P.as_tuple() == (2.0, 4.0, 0.5, 5.0, 0.5, 0.0, 1.0, 2.0, 1.0, 0.5)


def test_grid_nyquist_conventions():
    g = orc.make_grid(8, 0.5)
    k = 2 * np.pi * np.fft.fftfreq(8, 0.5)
    assert g.kx[0, 4] == 0.0 and g.ky[4, 0] == 0.0          # core_shell.jl:20
    assert np.isclose(g.k2[0, 4], k[4] ** 2)                 # core_shell.jl:23 keeps the Nyquist
    g7 = orc.make_grid(7, 1.0)
    assert np.count_nonzero(g7.kx == 0.0) == 1                 # odd n: only k = 0 vanishes


def test_variational_derivative():
    # checks.jl:7-11: central FD of the energy along a random direction vs sum(mu v)
    c, phi, grid, shape = setup64()
    v = np.random.default_rng(8).standard_normal(c.shape)
    eps = 1e-6
    num = (orc.energy(c + eps * v, shape, grid, P) - orc.energy(c - eps * v, shape, grid, P)) / (2 * eps)
    ana = np.sum(orc.chemical_potential(c, shape, grid, P) * v)
    assert np.isclose(num, ana, rtol=1e-6, atol=1e-6)


def test_dissipation_identity_and_conservation():
    # checks.jl:12-14
    c, phi, grid, shape = setup64()
    rate, diss = orc.transport_rate(c, shape, grid, P)
    dcdt = np.real(np.fft.ifft2(rate))
    assert np.isclose(np.sum(orc.chemical_potential(c, shape, grid, P) * dcdt), -diss, rtol=1e-10)
    assert abs(np.sum(dcdt)) < 1e-10


def test_initial_energy_known_answers():
    # check-results.txt:2 and :7 give E(t=0) = 329.48858453024934 (64^2, R=16) and
    # 4406.5104552251505 (256^2, R=70) for the MersenneTwister noise; across
    # PCG64 seeds the oracle's E0 has std 0.018 (64^2) and 0.081 (256^2).
    for seed in (5749, 1, 2):
        c, phi = orc.initial_fields(64, radius=16.0, seed=seed)
        e = orc.energy(c, orc.geometry(phi, P), orc.make_grid(64, 1.0), P)
        assert abs(e - 329.48858453024934) < 5 * 0.018
    c, phi = orc.initial_fields(256)
    e = orc.energy(c, orc.geometry(phi, P), orc.make_grid(256, 1.0), P)
    assert abs(e - 4406.5104552251505) < 5 * 0.081


def test_time_refinement_mass_and_energy():
    # checks.jl:17-25 with check-results.txt:2-6: mass drift < 1e-12, energy
    # non-increasing (1e-8), final-field RMS differences halving with dt.
    c, phi, _, _ = setup64()
    finals = []
    for dt in (0.01, 0.005, 0.0025):
        final, hist = orc.run_simulation(c, phi, dt=dt, steps=round(10 / dt))
        assert np.max(np.abs(hist[:, 1] - c.mean())) < 1e-12
        assert np.max(np.diff(hist[:, 2])) < 1e-8
        assert abs(hist[0, 2] - 329.48858453024934) < 5 * 0.018
        assert 0.0 < final.min() < final.max() < 1.0
        finals.append(final)
    r1 = np.sqrt(np.mean((finals[0] - finals[1]) ** 2))
    r2 = np.sqrt(np.mean((finals[1] - finals[2]) ** 2))
    # reference: 2.027e-4 and 1.023e-4 (ratio 1.98); first order in dt
    assert 1e-4 < r1 < 5e-4 and 5e-5 < r2 < 2.5e-4
    assert 1.7 < r1 / r2 < 2.3


def test_history_layout_and_record_then_step():
    c, phi, _, _ = setup64()
    c1, h1 = orc.run_simulation(c, phi, dt=0.01, steps=1)
    c0, h0 = orc.run_simulation(c, phi, dt=0.01, steps=0)
    assert h0.shape == (1, 6) and np.array_equal(c0, c)
    assert np.array_equal(h1[0], h0[0])                   # row 0 is the initial field
    assert h1[1, 0] == 0.01 and np.isclose(h1[1, 1], c.mean(), rtol=0, atol=1e-14)


def test_nonfinite_raises_with_step():
    c, phi, _, _ = setup64()
    bad = c.copy()
    bad[3, 5] = np.nan
    with pytest.raises(orc.NonFiniteError) as ei:
        orc.run_simulation(bad, phi, dt=0.01, steps=3)
    assert ei.value.step == 0


@pytest.mark.parametrize("name", ["disc16_r4", "disc48_r12", "disc64_r16", "disc96_r24_dt005"])
def test_oracle_matches_golden(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    p = orc.Parameters(*d["params"])
    c, h = orc.run_simulation(d["c0"], d["phi"], dt=float(d["dt"]), steps=int(d["steps"]), p=p)
    assert np.max(np.abs(c - d["c"])) <= 1e-13
    assert np.max(np.abs(h - d["history"]) / np.maximum(np.abs(d["history"]), 1e-300)) <= 1e-12
