"""The CPU oracle of the coupled c-phi model (original/2023-3d restated in
oracle/coupled_oracle.py): its stencil, its conservation, its stop rules, the
reference's dy/dz quirk, and a committed fixture that pins it against drift.
The library's coupled kernels are held to this oracle in test_gpu_coupled.py."""
import os

import numpy as np
import pytest

from oracle import coupled_oracle as co

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "coupled_24x16x32.npz")


def test_fourth_order_difference_is_the_modified_wavenumber():
    """D f = IFFT(i (8 sin(k h) - sin(2 k h)) / (6 h) FFT f): the periodic stencil of
    EvoKernels.h:125 is diagonal in Fourier space with that symbol."""
    f = np.random.default_rng(1).random((16, 12, 8))
    for ax, n, h in ((0, 16, 1.0), (1, 12, 0.7), (2, 8, 1.3)):
        k = 2 * np.pi * np.fft.fftfreq(n, h)
        s = (8 * np.sin(k * h) - np.sin(2 * k * h)) / (6 * h)
        shape = [1, 1, 1]
        shape[ax] = n
        spec = np.fft.ifftn(1j * s.reshape(shape) * np.fft.fftn(f)).real
        assert np.max(np.abs(spec - co.fd4(f, ax, h))) < 1e-13


def test_divergence_sums_to_zero_and_mass_is_conserved():
    c0, phi0 = co.initial_fields(16, 16, 16, 5.0, seed=3)
    M = co.local_terms(c0, phi0, co.CoupledParameters())[2]
    div = co.divergence(np.sin(np.arange(c0.size).reshape(c0.shape) * 0.37), M, (1.0, 1.0, 1.0))
    assert abs(div.sum()) < 1e-12
    c, phi, h, done, reason = co.run(c0, phi0, co.CoupledParameters(), 0.01, 30)
    assert done == 30 and reason == co.RUNNING
    assert np.max(np.abs(h[:, 1] - h[0, 1])) < 1e-14


def test_local_terms_are_the_derivatives_of_the_free_energy():
    """df/dc and df/dphi of EvoKernels.h:19-33 are the partial derivatives of
    f = (1-h)(A(c-ca)^2 + A0) + h B (c-cb1)^2 (c-cb2)^2 + P (1 - chi c) g."""
    p = co.CoupledParameters()

    def f(c, ph):
        h = ph ** 3 * (10 - 15 * ph + 6 * ph ** 2)
        g = ph ** 2 * (1 - ph) ** 2
        return ((1 - h) * (p.A * (c - p.ca) ** 2 + p.A0) + h * p.B * (c - p.cb1) ** 2 * (c - p.cb2) ** 2
                + p.P * (1 - p.chi * c) * g)

    rng = np.random.default_rng(2)
    c, ph = rng.uniform(-0.2, 1.2, 50), rng.uniform(0, 1, 50)
    dfdc, dfdphi, M = co.local_terms(c, ph, p)
    e = 1e-6
    assert np.max(np.abs(dfdc - (f(c + e, ph) - f(c - e, ph)) / (2 * e))) < 1e-7
    assert np.max(np.abs(dfdphi - (f(c, ph + e) - f(c, ph - e)) / (2 * e))) < 1e-7
    assert np.allclose(M, p.mobility * ph ** 3 * (10 - 15 * ph + 6 * ph ** 2))


def test_z_gradient_spacing_quirk():
    """The reference passes dy to the z-gradient of mu (evolve.cu:124): the same
    result when dy == dz, a different one otherwise."""
    c0, phi0 = co.initial_fields(12, 12, 16, 4.0, seed=4)
    p = co.CoupledParameters()
    a = co.run(c0, phi0, p, 0.01, 3, spacing=(1.0, 1.0, 1.0), z_grad_spacing="dy")[0]
    b = co.run(c0, phi0, p, 0.01, 3, spacing=(1.0, 1.0, 1.0), z_grad_spacing="dz")[0]
    assert np.array_equal(a, b)
    a = co.run(c0, phi0, p, 0.01, 3, spacing=(1.0, 0.8, 1.2), z_grad_spacing="dy")[0]
    b = co.run(c0, phi0, p, 0.01, 3, spacing=(1.0, 0.8, 1.2), z_grad_spacing="dz")[0]
    assert np.max(np.abs(a - b)) > 1e-9


def test_stop_rules():
    c0, phi0 = co.initial_fields(12, 12, 12, 4.0, seed=5)
    p = co.CoupledParameters()
    # convergence: max|dc| <= tolerance after the first step
    c, phi, h, done, reason = co.run(c0, phi0, p, 0.01, 10, tolerance=1.0)
    assert (done, reason) == (1, co.CONVERGED) and h.shape == (2, 6)
    # mass check that always fails: the fields of the failing step are not kept
    c, phi, h, done, reason = co.run(c0, phi0, p, 0.01, 10, comperr=-1.0)
    assert (done, reason) == (0, co.MASS_ERROR)
    assert np.array_equal(c, c0) and np.array_equal(phi, phi0)
    # composition outside [-0.4, 1.4]
    cb = c0.copy()
    cb[0, 0, 0] = 1.6
    c, phi, h, done, reason = co.run(cb, phi0, p, 0.01, 10)
    assert (done, reason) == (1, co.OUT_OF_BOUNDS)


def test_golden_fixture():
    """The oracle reproduces its committed fixture (tests/golden/make_golden.py)."""
    g = np.load(GOLDEN)
    p = co.CoupledParameters(**{k: float(v) for k, v in zip(g["param_names"], g["param_values"])})
    c, phi, h, done, reason = co.run(g["c0"], g["phi0"], p, float(g["dt"]), int(g["steps"]),
                                     spacing=tuple(g["spacing"]))
    assert done == int(g["steps"])
    assert np.max(np.abs(c - g["c"])) < 1e-13
    assert np.max(np.abs(phi - g["phi"])) < 1e-13
    assert np.max(np.abs(h - g["history"])) < 1e-13
