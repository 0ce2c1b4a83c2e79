"""GPU adjoint (esc_adjoint through the C ABI) against the CPU oracle.

Checks, on small grids and in FP64: the loss, dL/dc0 and dL/d(P, chi, kappa, M0)
against the oracle's reverse mode; the directional derivative against the
oracle's forward (dual-number) mode; parameter gradients against central
finite differences (h = 1e-4, FP64) of the GPU forward itself.
"""
import numpy as np
import pytest

import esc
from oracle import adjoint_oracle as adj
from oracle import core_shell_oracle as orc

pytestmark = pytest.mark.gpu


def _case(n, steps, seed=3):
    p = orc.Parameters()
    c0, phi = orc.initial_fields(n, radius=n / 4, width=2.0, seed=seed)
    pt = adj._with(p, P=p.P * 1.1, chi=p.chi * 0.9)           # target: perturbed (P, chi)
    ct = adj.forward_states(c0, phi, steps, 0.01, pt)[-1]
    return p, c0, phi, ct


def _ep(p):
    return esc.Parameters(A=p.A, B=p.B, chi=p.chi, P=p.P, ca=p.ca, cb=p.cb, cc=p.cc, kappa=p.kappa,
                          mobility=p.mobility, Q=p.Q)


@pytest.mark.parametrize("n,steps,K", [(32, 30, 7), (64, 45, 0), (48, 20, 20)])
def test_adjoint_matches_oracle(n, steps, K):
    p, c0, phi, ct = _case(n, steps)
    lamF = 1e-3
    Lo, go, tho = adj.gradient(c0, phi, steps, 0.01, ct, lamF, p)
    with esc.Context(phi, p=_ep(p)) as ctx:
        L, g, th = ctx.adjoint(c0, ct, dt=0.01, steps=steps, lambda_F=lamF, ckpt_every=K)
    assert abs(L - Lo) <= 1e-12 * abs(Lo)
    assert np.max(np.abs(g - go)) <= 1e-10 * np.max(np.abs(go))
    assert np.max(np.abs(th - tho) / np.maximum(np.abs(tho), 1e-30)) <= 1e-9, (th, tho)


def test_adjoint_directional_derivative_vs_dual_numbers():
    n, steps = 64, 40
    p, c0, phi, ct = _case(n, steps, seed=8)
    rng = np.random.default_rng(8)
    v = rng.standard_normal(c0.shape)
    th_dir = rng.standard_normal(4)
    jv = adj.jvp(c0, phi, steps, 0.01, ct, 1e-3, p, v, th_dir)
    with esc.Context(phi, p=_ep(p)) as ctx:
        _, g, th = ctx.adjoint(c0, ct, dt=0.01, steps=steps, lambda_F=1e-3)
    ad = float(np.sum(g * v) + np.dot(th, th_dir))
    assert abs(ad - jv) <= 1e-9 * abs(jv)


def test_adjoint_parameters_vs_central_differences():
    n, steps, lamF, h = 64, 40, 1e-3, 1e-4
    p, c0, phi, ct = _case(n, steps, seed=5)

    def gpu_loss(pp):
        c, hist = esc.run_simulation(c0, phi, dt=0.01, steps=steps, p=_ep(pp))
        return 0.5 * float(np.sum((c - ct) ** 2)) + lamF * hist[-1, 2]

    with esc.Context(phi, p=_ep(p)) as ctx:
        _, _, th = ctx.adjoint(c0, ct, dt=0.01, steps=steps, lambda_F=lamF)
    tol = {0: 1e-6, 1: 1e-6, 2: 1e-4, 3: 1e-5}
    for k in range(4):
        fd = (gpu_loss(adj.perturbed(p, k, h)) - gpu_loss(adj.perturbed(p, k, -h))) / (2 * h)
        assert abs(fd - th[k]) <= tol[k] * max(abs(fd), 1e-12), (adj.THETA[k], fd, th[k])


def test_adjoint_mixed_precision_close_to_fp64():
    n, steps = 64, 40
    p, c0, phi, ct = _case(n, steps)
    with esc.Context(phi, p=_ep(p)) as c64:
        L64, g64, th64 = c64.adjoint(c0, ct, dt=0.01, steps=steps)
    with esc.Context(phi, p=_ep(p), precision="mixed") as c32:
        L32, g32, th32 = c32.adjoint(c0, ct, dt=0.01, steps=steps)
    assert abs(L32 - L64) <= 1e-6 * abs(L64)
    assert np.max(np.abs(g32 - g64)) <= 1e-4 * np.max(np.abs(g64))
    assert np.max(np.abs(th32 - th64) / np.abs(th64)) <= 1e-3


def test_batch_adjoint_matches_oracle_per_particle():
    """esc_batch_adjoint: every particle of a one-size batch gets its own oracle gradient."""
    n, steps, lamF = 48, 25, 1e-3
    base = orc.Parameters()
    ps = [adj._with(base, P=base.P * f, chi=base.chi * g, kappa=base.kappa * k)
          for f, g, k in [(1.0, 1.0, 1.0), (1.3, 0.8, 1.2), (0.7, 1.2, 0.9)]]
    c0s, phis, cts = [], [], []
    for i, p in enumerate(ps):
        c0, phi = orc.initial_fields(n, radius=n / 4 + i, width=2.0, seed=20 + i)
        pt = adj._with(p, P=p.P * 1.1, chi=p.chi * 0.9)
        c0s.append(c0)
        phis.append(phi)
        cts.append(adj.forward_states(c0, phi, steps, 0.01, pt)[-1])
    with esc.Batch(phis, params=[_ep(p) for p in ps], precision="fp64") as b:
        L, gs, th = b.adjoint(c0s, cts, dt=0.01, steps=steps, lambda_F=lamF, ckpt_every=6)
    for i, p in enumerate(ps):
        Lo, go, tho = adj.gradient(c0s[i], phis[i], steps, 0.01, cts[i], lamF, p)
        assert abs(L[i] - Lo) <= 1e-12 * abs(Lo)
        assert np.max(np.abs(gs[i] - go)) <= 1e-10 * np.max(np.abs(go))
        assert np.max(np.abs(th[i] - tho) / np.maximum(np.abs(tho), 1e-30)) <= 1e-9, (i, th[i], tho)


def test_batch_adjoint_rejects_mixed_sizes():
    phis = [orc.particle_disc(32, 1.0, 8.0, 2.0), orc.particle_disc(48, 1.0, 12.0, 2.0)]
    c0s = [orc.interior_noise(f, 1) for f in phis]
    with esc.Batch(phis, precision="fp64") as b:
        with pytest.raises(esc.EscError):
            b.adjoint(c0s, c0s, steps=3)


@pytest.mark.parametrize("n,steps", [(256, 30), (512, 20)])
def test_batch_adjoint_mixed_close_to_fp64(n, steps):
    """Mixed contexts run the mixed adjoint step (FP64 adjoint state, FP32 derived-field
    transforms): at the bench's grid sizes its batched gradients stay within the tolerances
    of the single-particle mixed test of the FP64 gradients."""
    lamF = 1e-3
    base = orc.Parameters()
    ps = [adj._with(base, P=base.P * f, chi=base.chi * g) for f, g in [(1.0, 1.0), (1.4, 0.8), (0.7, 1.3)]]
    c0s, phis, cts = [], [], []
    for i, p in enumerate(ps):
        c0, phi = orc.initial_fields(n, radius=0.3 * n, width=2.0, seed=40 + i)
        c0s.append(c0)
        phis.append(phi)
    with esc.Batch(phis, params=[_ep(adj._with(p, P=p.P * 1.1, chi=p.chi * 0.9)) for p in ps],
                   precision="fp64") as bt:
        cts, _, _ = bt.run(c0s, dt=0.01, steps=steps, with_history=False)
    out = {}
    for prec in ("fp64", "mixed"):
        with esc.Batch(phis, params=[_ep(p) for p in ps], precision=prec) as b:
            out[prec] = b.adjoint(c0s, cts, dt=0.01, steps=steps, lambda_F=lamF, ckpt_every=7)
    L64, g64, th64 = out["fp64"]
    L32, g32, th32 = out["mixed"]
    for i in range(len(ps)):
        assert abs(L32[i] - L64[i]) <= 1e-6 * abs(L64[i])
        assert np.max(np.abs(g32[i] - g64[i])) <= 1e-4 * np.max(np.abs(g64[i]))
        assert np.max(np.abs(np.asarray(th32[i]) - th64[i]) / np.abs(th64[i])) <= 1e-3, (i, th32[i], th64[i])
