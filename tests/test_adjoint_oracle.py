"""The gradient oracle pinned against itself three ways on the CPU: reverse mode
(transposed step) == forward mode (dual numbers through the reference step)
to rounding, and both == central finite differences of the reference loss."""
import numpy as np

from oracle import adjoint_oracle as adj
from oracle import core_shell_oracle as orc


def _case(n=24, steps=15):
    p = orc.Parameters()
    c0, phi = orc.initial_fields(n, radius=6.0, width=2.0, seed=4)
    ct = adj.forward_states(c0, phi, steps, 0.01, adj._with(p, P=5.5, chi=0.45))[-1]
    return p, c0, phi, ct, steps


def test_reverse_equals_forward_mode():
    p, c0, phi, ct, steps = _case()
    L, g, th = adj.gradient(c0, phi, steps, 0.01, ct, 1e-3, p)
    rng = np.random.default_rng(2)
    v, d = rng.standard_normal(c0.shape), rng.standard_normal(4)
    jv = adj.jvp(c0, phi, steps, 0.01, ct, 1e-3, p, v, d)
    assert abs(float(np.sum(g * v) + np.dot(th, d)) - jv) <= 1e-12 * abs(jv)
    assert abs(L - adj.loss(c0, phi, steps, 0.01, ct, 1e-3, p)) <= 1e-14 * abs(L)


def test_reverse_mode_vs_central_differences():
    p, c0, phi, ct, steps = _case()
    _, g, th = adj.gradient(c0, phi, steps, 0.01, ct, 1e-3, p)
    for k, tol in zip(range(4), (1e-8, 1e-8, 1e-5, 1e-6)):
        h = 1e-4
        fd = (adj.loss(c0, phi, steps, 0.01, ct, 1e-3, adj.perturbed(p, k, h))
              - adj.loss(c0, phi, steps, 0.01, ct, 1e-3, adj.perturbed(p, k, -h))) / (2 * h)
        assert abs(fd - th[k]) <= tol * abs(fd)
    v = np.random.default_rng(3).standard_normal(c0.shape)
    h = 1e-6
    fd = (adj.loss(c0 + h * v, phi, steps, 0.01, ct, 1e-3, p) - adj.loss(c0 - h * v, phi, steps, 0.01, ct, 1e-3, p)) / (2 * h)
    assert abs(fd - float(np.sum(g * v))) <= 1e-6 * abs(fd)
