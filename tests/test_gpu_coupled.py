"""The coupled c-phi model on the GPU (esc_cphi_*, csrc/esc_cphi.cuh) against the
CPU oracle of original/2023-3d (oracle/coupled_oracle.py), in FP64.

Parity: c, phi and the history within 1e-12 (relative to the field's maximum)
on cubic and non-cubic grids, unequal spacings, the reference's constants and
others; the stop rules of the reference's loop (convergence, composition
bounds, the mass check) and the non-finite path give the oracle's step and
reason; host and device entry points agree."""
import numpy as np
import pytest

from oracle import coupled_oracle as co

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def hist_rel(h, ho):
    out = 0.0
    for j in range(6):
        scale = max(np.max(np.abs(ho[:, j])), 1e-300)
        out = max(out, float(np.max(np.abs(h[:, j] - ho[:, j])) / scale))
    return out


def run_both(shape, spacing, steps, p=co.CoupledParameters(), seed=1, radius=None, dt=0.01, **kw):
    from esc import coupled
    radius = radius or 0.3 * min(shape)
    c0, phi0 = co.initial_fields(*shape, radius, seed=seed, p=p)
    pp = coupled.CoupledParameters(**vars(p))
    c, phi, h, done, reason = coupled.run_coupled(c0, phi0, dt=dt, steps=steps, spacing=spacing, params=pp, **kw)
    co_, pho, ho, doneo, reasono = co.run(c0, phi0, p, dt, steps, spacing=spacing, **kw)
    return (c, phi, h, done, reason), (co_, pho, ho, doneo, reasono)


@pytest.mark.parametrize("shape,spacing,steps", [
    ((16, 16, 16), (1.0, 1.0, 1.0), 40),
    ((24, 16, 32), (1.0, 0.9, 1.1), 25),
    ((32, 24, 48), (1.0, 1.0, 1.0), 20),
    ((8, 12, 64), (0.8, 1.0, 1.2), 15),
    ((64, 64, 64), (1.0, 1.0, 1.0), 10),
    # the eight-element 128- and 256-point plans on every axis (the plans of the 256^3 bench)
    ((8, 128, 256), (1.0, 1.0, 1.0), 6),
    ((256, 16, 128), (1.0, 1.1, 0.9), 6),
])
def test_coupled_matches_oracle(shape, spacing, steps):
    (c, phi, h, done, reason), (co_, pho, ho, doneo, reasono) = run_both(shape, spacing, steps)
    assert (done, reason) == (doneo, reasono) == (steps, 0)
    assert rel(c, co_) < RTOL, rel(c, co_)
    assert rel(phi, pho) < RTOL, rel(phi, pho)
    assert hist_rel(h, ho) < 1e-11, hist_rel(h, ho)
    assert np.max(np.abs(h[:, 1] - h[0, 1])) < 1e-13  # mass


def test_coupled_other_constants_and_fixture():
    from esc import coupled
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "coupled_24x16x32.npz"))
    p = coupled.CoupledParameters(**{k: float(v) for k, v in zip(g["param_names"], g["param_values"])})
    c, phi, h, done, reason = coupled.run_coupled(g["c0"], g["phi0"], dt=float(g["dt"]), steps=int(g["steps"]),
                                                  spacing=tuple(g["spacing"]), params=p)
    assert rel(c, g["c"]) < RTOL and rel(phi, g["phi"]) < RTOL
    assert hist_rel(h, g["history"]) < 1e-11


def test_coupled_long_run_crosses_graph_chunks():
    """45 steps = 32 + 8 + 4 + 1 captured chunks."""
    (c, phi, h, done, reason), (co_, pho, ho, _, _) = run_both((16, 24, 16), (1.0, 1.0, 1.0), 45,
                                                               p=co.CoupledParameters(relax=0.05, kappa_phi=4.0))
    assert done == 45
    assert rel(c, co_) < RTOL and rel(phi, pho) < RTOL
    assert hist_rel(h, ho) < 1e-11


def test_coupled_convergence_stop():
    (c, phi, h, done, reason), (co_, pho, ho, doneo, reasono) = run_both((16, 16, 16), (1, 1, 1), 50,
                                                                         tolerance=2e-3)
    assert reasono == co.CONVERGED and (done, reason) == (doneo, reasono)
    assert rel(c, co_) < RTOL
    assert np.all(h[done + 1:] == 0.0)


def test_coupled_bounds_stop():
    from esc import coupled
    p = co.CoupledParameters()
    c0, phi0 = co.initial_fields(16, 16, 16, 5.0, seed=2, p=p)
    c0[3, 4, 5] = 1.6
    c, phi, h, done, reason = coupled.run_coupled(c0, phi0, dt=0.01, steps=10)
    co_, pho, ho, doneo, reasono = co.run(c0, phi0, p, 0.01, 10)
    assert (done, reason) == (doneo, reasono) == (1, co.OUT_OF_BOUNDS)
    assert rel(c, co_) < RTOL


def test_coupled_mass_error_keeps_the_input():
    from esc import coupled
    c0, phi0 = co.initial_fields(16, 16, 16, 5.0, seed=2)
    with pytest.raises(coupled.MassError) as e:
        coupled.run_coupled(c0, phi0, dt=0.01, steps=10, comperr=-1.0)
    assert e.value.step == 0
    # the context stays usable and returns the input fields unchanged on the failing call
    with coupled.Coupled((16, 16, 16)) as ctx:
        with pytest.raises(coupled.MassError):
            ctx.run(c0, phi0, steps=3, comperr=-1.0)
        c, phi, h, done, reason = ctx.run(c0, phi0, steps=3)
        assert done == 3
        co_ = co.run(c0, phi0, co.CoupledParameters(), 0.01, 3)[0]
        assert rel(c, co_) < RTOL


def test_coupled_nonfinite_input():
    from esc import NonFiniteError, coupled
    c0, phi0 = co.initial_fields(16, 16, 16, 5.0, seed=2)
    c0[1, 2, 3] = np.nan
    with pytest.raises(NonFiniteError) as e:
        coupled.run_coupled(c0, phi0, steps=4)
    assert e.value.step == 0


def test_coupled_device_entry_point_matches_host():
    import torch
    from esc import coupled
    c0, phi0 = co.initial_fields(24, 16, 32, 6.0, seed=9)
    with coupled.Coupled(c0.shape) as ctx:
        c, phi, h, done, reason = ctx.run(c0, phi0, steps=12)
        dc, dp = torch.from_numpy(c0).cuda(), torch.from_numpy(phi0).cuda()
        dh = torch.zeros(6 * 13, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        done_d, reason_d = ctx.run_device(dc.data_ptr(), dp.data_ptr(), 12, 0.01, hist_ptr=dh.data_ptr())
        assert (done_d, reason_d) == (done, reason) == (12, 0)
        assert np.array_equal(dc.cpu().numpy(), c) and np.array_equal(dp.cpu().numpy(), phi)
        assert np.array_equal(dh.cpu().numpy().reshape(6, 13).T, h)


def test_coupled_rejects_bad_arguments():
    from esc import EscError, coupled
    with pytest.raises(EscError):
        coupled.Coupled((10, 16, 16))
    with pytest.raises(EscError):
        coupled.Coupled((16, 16, 16), spacing=(1.0, 0.0, 1.0))
    assert coupled.supported_axis(256) and not coupled.supported_axis(1024)


def test_coupled_and_planar_runs_share_a_process():
    """A 2-D run and a coupled run of the same grid size in one process, in both
    orders: each keeps its own twiddle tables (the coupled kernel units must not
    share kernel or table symbols with the 2-D units of the same size)."""
    import esc
    from esc import coupled
    from oracle import core_shell_oracle as orc
    c2, phi2 = orc.initial_fields(64, radius=16.0)
    c3, phi3 = co.initial_fields(64, 64, 64, 18.0, seed=3)
    ref2, _ = orc.run_simulation(c2, phi2, dt=0.01, steps=5)
    ref3 = co.run(c3, phi3, co.CoupledParameters(), 0.01, 3)[0]
    for _ in range(2):
        a, _ = esc.run_simulation(c2, phi2, dt=0.01, steps=5)
        b = coupled.run_coupled(c3, phi3, dt=0.01, steps=3)[0]
        assert rel(a, ref2) < RTOL and rel(b, ref3) < RTOL
