"""The CPU oracle pinned against the reference's own checks and known answers.

The reference's test file checks.jl (30 lines) asserts physics identities and
run properties; check-results.txt records the numbers one run of it printed.
The oracle draws the reference's own noise (Julia's MersenneTwister stream,
restated in oracle/julia_rng.py), so those numbers are pinned here as known
answers: energies, composition ranges and RMS differences to ~1e-10 relative,
and the identities exactly as checks.jl asserts them.
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


# Known answers printed by the reference's checks.jl (check-results.txt:2-7):
# dt -> (energy at t=0, energy at t=10, min c, max c) for 64^2, radius 16, seed 5749
KNOWN_64 = {
    0.01: (329.48858453024934, 290.1672693863404, 0.03738467482348276, 0.9430096320792813),
    0.005: (329.48858453024934, 290.15644231050993, 0.037201502506359285, 0.9430283569784008),
    0.0025: (329.48858453024934, 290.1511266046432, 0.037106495159182185, 0.9430402849426585),
}
KNOWN_RMS = (0.0002027456340109754, 0.00010231034501867524)     # check-results.txt:5-6
KNOWN_256 = (4406.5104552251505, 3592.0207507163714, 0.007360143442235456, 0.9899654270279202)  # :7
RTOL_KNOWN = 1e-10


def relerr(a, b):
    return abs(a - b) / abs(b)


def test_initial_energy_known_answers():
    # check-results.txt:2 and :7: E(t=0) for initial_fields(64; radius=16) and initial_fields(256)
    c, phi = orc.initial_fields(64, radius=16.0)
    e = orc.energy(c, orc.geometry(phi, P), orc.make_grid(64, 1.0), P)
    assert relerr(e, KNOWN_64[0.01][0]) <= 1e-14
    c, phi = orc.initial_fields(256)
    e = orc.energy(c, orc.geometry(phi, P), orc.make_grid(256, 1.0), P)
    assert relerr(e, KNOWN_256[0]) <= 1e-14


def test_time_refinement_known_answers():
    # checks.jl:17-25 with check-results.txt:2-6: mass drift < 1e-12, energy
    # non-increasing (1e-8), and the recorded energies, ranges and RMS differences.
    c, phi, _, _ = setup64()
    finals = []
    for dt in (0.01, 0.005, 0.0025):
        final, hist = orc.run_simulation(c, phi, dt=dt, steps=round(10 / dt))
        assert np.max(np.abs(hist[:, 1] - c.mean())) < 1e-12
        assert np.max(np.diff(hist[:, 2])) < 1e-8
        e0, e1, lo, hi = KNOWN_64[dt]
        assert relerr(hist[0, 2], e0) <= 1e-14
        assert relerr(hist[-1, 2], e1) <= RTOL_KNOWN
        assert relerr(final.min(), lo) <= RTOL_KNOWN and relerr(final.max(), hi) <= RTOL_KNOWN
        finals.append(final)
    r1 = np.sqrt(np.mean((finals[0] - finals[1]) ** 2))
    r2 = np.sqrt(np.mean((finals[1] - finals[2]) ** 2))
    # the RMS of a difference of two fields: its relative error is ~1e4 times c's
    assert relerr(r1, KNOWN_RMS[0]) <= 1e-9 and relerr(r2, KNOWN_RMS[1]) <= 1e-9


def test_default_example_known_answers():
    # checks.jl:26-30 with check-results.txt:7: the default 256^2 example over 1000 steps
    orc.set_workers(os.cpu_count() or 1)
    try:
        c, phi = orc.initial_fields(256)
        final, hist = orc.run_simulation(c, phi, dt=0.01, steps=1000)
    finally:
        orc.set_workers(1)
    assert np.max(np.abs(hist[:, 1] - c.mean())) < 1e-12
    assert np.max(np.diff(hist[:, 2])) < 1e-8
    e0, e1, lo, hi = KNOWN_256
    assert relerr(hist[0, 2], e0) <= 1e-14 and relerr(hist[-1, 2], e1) <= RTOL_KNOWN
    assert relerr(final.min(), lo) <= RTOL_KNOWN and relerr(final.max(), hi) <= RTOL_KNOWN


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
