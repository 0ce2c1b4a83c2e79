"""Cluster-resident runs of single small FP64 grids (csrc/esc_cluster.cu).

A single 128^2 or 256^2 FP64 context can run its whole time loop in one launch
of one thread-block cluster, the state in distributed shared memory; at creation
the library times that path against the launch-per-phase path and keeps the
faster (ESC_CLUSTER=1 forces the cluster path, 0 forbids it).  These tests force
the cluster path and hold it to the CPU oracle (core_shell.jl:84-103 restated) at
1e-12 and to the launch-per-phase path at the rounding level, and check its
non-finite stop, its queued device-memory entry points and its history."""
import numpy as np
import pytest

import esc
from oracle import core_shell_oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _force_cluster(monkeypatch):
    monkeypatch.setenv("ESC_CLUSTER", "1")

RTOL = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def hist_rel(h, ho):
    return max(float(np.max(np.abs(h[:, j] - ho[:, j])) / max(np.max(np.abs(ho[:, j])), 1e-300)) for j in range(6))


@pytest.mark.parametrize("n,steps", [(128, 45), (256, 40)])
def test_cluster_path_matches_oracle(n, steps):
    c0, phi = orc.initial_fields(n, radius=0.3 * n, width=2.0, seed=17)
    with esc.Context(phi) as ctx:
        if not ctx.uses_cluster:
            pytest.skip("this device cannot place the cluster")
        c, h = ctx.run(c0, dt=0.01, steps=steps)
    co, ho = orc.run_simulation(c0, phi, dt=0.01, steps=steps)
    assert rel(c, co) < RTOL, rel(c, co)
    assert hist_rel(h, ho) < RTOL, hist_rel(h, ho)


@pytest.mark.parametrize("n", [128, 256])
def test_cluster_path_agrees_with_launch_per_phase(n, monkeypatch):
    c0, phi = orc.initial_fields(n, radius=0.35 * n, width=4.0, seed=5)
    p = esc.Parameters(P=6.0, kappa=3.0)
    with esc.Context(phi, p=p) as ctx:
        if not ctx.uses_cluster:
            pytest.skip("this device cannot place the cluster")
        c1, h1 = ctx.run(c0, dt=0.01, steps=100)
    monkeypatch.setenv("ESC_CLUSTER", "0")
    with esc.Context(phi, p=p) as ctx:
        assert not ctx.uses_cluster
        c2, h2 = ctx.run(c0, dt=0.01, steps=100)
    assert rel(c1, c2) < RTOL and hist_rel(h1, h2) < RTOL


def test_cluster_path_nonfinite_stops_and_keeps_c():
    c0, phi = orc.initial_fields(256, radius=70.0, width=4.0, seed=3)
    c0[10, 20] = np.nan
    with esc.Context(phi) as ctx:
        if not ctx.uses_cluster:
            pytest.skip("this device cannot place the cluster")
        cin = c0.copy()
        with pytest.raises(esc.NonFiniteError) as e:
            ctx.run(cin, dt=0.01, steps=10)
        assert e.value.step == 0
        # the context stays usable
        c1, _ = ctx.run(np.nan_to_num(c0, nan=0.5), dt=0.01, steps=3)
        assert np.all(np.isfinite(c1))


def test_cluster_path_queued_device_run():
    import torch
    c0, phi = orc.initial_fields(128, radius=40.0, width=2.0, seed=8)
    with esc.Context(phi) as ctx:
        if not ctx.uses_cluster:
            pytest.skip("this device cannot place the cluster")
        c, h = ctx.run(c0, dt=0.01, steps=33)
        d = torch.from_numpy(c0).cuda()
        dh = torch.zeros(6 * 34, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        ctx.run_device_async(d.data_ptr(), 33, 0.01, dh.data_ptr())
        ctx.wait()
        assert np.array_equal(d.cpu().numpy(), c)
        assert np.array_equal(dh.cpu().numpy().reshape(6, 34).T, h)


@pytest.mark.parametrize("n", [128, 256])
def test_timed_choice_gives_oracle_results(n, monkeypatch):
    """Unforced, the creation times both paths and keeps the faster; either way the
    results are the oracle's."""
    monkeypatch.delenv("ESC_CLUSTER", raising=False)
    c0, phi = orc.initial_fields(n, radius=0.3 * n, width=2.0, seed=23)
    with esc.Context(phi) as ctx:
        c, h = ctx.run(c0, dt=0.01, steps=12)
    co, ho = orc.run_simulation(c0, phi, dt=0.01, steps=12)
    assert rel(c, co) < RTOL and hist_rel(h, ho) < RTOL
