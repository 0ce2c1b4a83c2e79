"""GPU parity of the batched stepper (esc_batch_*): particles of different grid
sizes and parameters advanced together, each checked against the CPU oracle
(core_shell.jl:84-103 restated in oracle/core_shell_oracle.py) or against the
single-particle path.

The step counts cross the captured 32-step chunk (a graph launch per size group
plus single steps for the remainder), and the batches hold several size groups,
which run on their own streams.
"""
import numpy as np
import pytest

import esc
from oracle import core_shell_oracle as orc

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def hist_rel(h, ho):
    out = []
    for j in range(6):
        scale = max(np.max(np.abs(ho[:, j])), 1e-300)
        out.append(float(np.max(np.abs(h[:, j] - ho[:, j])) / scale))
    return max(out)


def particles(sizes, seed0=100):
    """(n, c0, phi, esc.Parameters, oracle Parameters) per particle, sampled around the defaults."""
    rng = np.random.default_rng(seed0)
    out = []
    for k, n in enumerate(sizes):
        c0, phi = orc.initial_fields(n, radius=0.3 * n, width=max(1.0, 4.0 * n / 256), seed=seed0 + k)
        p = esc.Parameters(P=5.0 * rng.uniform(0.5, 2.0), chi=0.5 * rng.uniform(0.5, 1.5),
                           kappa=2.0 * rng.uniform(0.5, 2.0))
        po = orc.Parameters(A=p.A, B=p.B, chi=p.chi, P=p.P, ca=p.ca, cb=p.cb, cc=p.cc, kappa=p.kappa,
                            mobility=p.mobility, Q=p.Q)
        out.append((n, c0, phi, p, po))
    return out


SIZES = [48, 64, 32, 96, 64, 128, 48, 192, 32]


def test_batch_fp64_matches_oracle_per_particle():
    parts = particles(SIZES)
    steps = 41
    with esc.Batch([x[2] for x in parts], params=[x[3] for x in parts], precision="fp64") as b:
        cs, hs, bad = b.run([x[1] for x in parts], dt=0.01, steps=steps)
    assert bad == [-1] * len(parts)
    for (n, c0, phi, p, po), c, h in zip(parts, cs, hs):
        co, ho = orc.run_simulation(c0, phi, dt=0.01, steps=steps, p=po)
        assert rel(c, co) < RTOL_FP64, n
        assert hist_rel(h, ho) < RTOL_FP64, n


def test_batch_mixed_within_bound_of_fp64():
    parts = particles(SIZES, seed0=300)
    steps = 70
    res = {}
    for prec in ("fp64", "mixed"):
        with esc.Batch([x[2] for x in parts], params=[x[3] for x in parts], precision=prec) as b:
            res[prec] = b.run([x[1] for x in parts], dt=0.01, steps=steps)
    for k in range(len(parts)):
        c64, h64 = res["fp64"][0][k], res["fp64"][1][k]
        c32, h32 = res["mixed"][0][k], res["mixed"][1][k]
        assert rel(c32, c64) < 1e-5
        assert np.max(np.abs(h32[:, 1] - h32[0, 1])) < 1e-12      # mass: FP64 state and reductions
        assert np.max(np.abs(h32[:, 2] - h64[:, 2])) / np.max(np.abs(h64[:, 2])) < 1e-5


def test_batch_equals_single_particle_runs():
    """A batch and one context per particle agree (the autotuner may pick other kernel families
    for a single particle, whose FFT plans round differently)."""
    parts = particles([64, 96, 64], seed0=500)
    steps = 35
    with esc.Batch([x[2] for x in parts], params=[x[3] for x in parts], precision="fp64") as b:
        cs, hs, _ = b.run([x[1] for x in parts], dt=0.01, steps=steps)
    for (n, c0, phi, p, po), c, h in zip(parts, cs, hs):
        c1, h1 = esc.run_simulation(c0, phi, dt=0.01, steps=steps, p=p)
        assert rel(c, c1) < RTOL_FP64
        assert hist_rel(h, h1) < RTOL_FP64


def test_batch_device_io_matches_host_io():
    import torch
    parts = particles([64, 128, 96, 64], seed0=700)
    steps = 40
    with esc.Batch([x[2] for x in parts], params=[x[3] for x in parts], precision="mixed") as b:
        cs, hs, _ = b.run([x[1] for x in parts], dt=0.01, steps=steps)
        work = [torch.from_numpy(x[1].copy()).cuda() for x in parts]
        hist = torch.zeros(len(parts) * 6 * (steps + 1), dtype=torch.float64, device="cuda")
        bad = b.run_device([w.data_ptr() for w in work], steps, 0.01, hist.data_ptr())
        torch.cuda.synchronize()
    assert bad == [-1] * len(parts)
    hd = hist.cpu().numpy().reshape(len(parts), 6, steps + 1)
    for k in range(len(parts)):
        assert np.array_equal(work[k].cpu().numpy(), cs[k])
        assert np.array_equal(hd[k].T, hs[k])


def test_batch_nonfinite_particle_is_isolated():
    """A non-finite field stops only its own particle (core_shell.jl:93 per instance): its step is
    reported, its c is left as it was, and the other particles, including those of its size group,
    are unaffected."""
    parts = particles([64, 64, 96, 128], seed0=900)
    c0s = [x[1].copy() for x in parts]
    c0s[1][5, 7] = np.nan
    steps = 40
    with esc.Batch([x[2] for x in parts], params=[x[3] for x in parts], precision="fp64") as b:
        cs, hs, bad = b.run(c0s, dt=0.01, steps=steps)
    assert bad[1] == 0
    assert bad[0] == bad[2] == bad[3] == -1
    assert np.array_equal(np.isnan(cs[1]), np.isnan(c0s[1]))
    assert np.array_equal(np.nan_to_num(cs[1]), np.nan_to_num(c0s[1]))
    for k in (0, 2, 3):
        n, c0, phi, p, po = parts[k]
        co, ho = orc.run_simulation(c0, phi, dt=0.01, steps=steps, p=po)
        assert rel(cs[k], co) < RTOL_FP64
        assert hist_rel(hs[k], ho) < RTOL_FP64


def test_batch_repeated_runs_restart_the_step_counter():
    """Each run starts its history at t = 0 and gives the same result (per-group step counters)."""
    parts = particles([64, 96], seed0=1100)
    with esc.Batch([x[2] for x in parts], params=[x[3] for x in parts], precision="mixed") as b:
        r1 = b.run([x[1] for x in parts], dt=0.01, steps=33)
        r2 = b.run([x[1] for x in parts], dt=0.01, steps=33)
    for k in range(len(parts)):
        assert np.array_equal(r1[0][k], r2[0][k])
        assert np.array_equal(r1[1][k], r2[1][k])
        assert np.allclose(r1[1][k][:, 0], 0.01 * np.arange(34), rtol=0, atol=1e-15)


def test_nonfinite_device_io_leaves_c_unchanged():
    """The device-memory paths keep the input field of a particle stopped on a non-finite value,
    as the host paths do (the single-particle drop-in and the batch)."""
    import torch
    parts = particles([64, 64], seed0=1300)
    c0s = [x[1].copy() for x in parts]
    c0s[0][3, 4] = np.inf
    with esc.Batch([x[2] for x in parts], params=[x[3] for x in parts], precision="mixed") as b:
        work = [torch.from_numpy(c).cuda() for c in c0s]
        bad = b.run_device([w.data_ptr() for w in work], 36, 0.01)
        torch.cuda.synchronize()
    assert bad == [0, -1]
    assert np.array_equal(work[0].cpu().numpy(), c0s[0])
    assert np.all(np.isfinite(work[1].cpu().numpy()))
    with esc.Context(parts[0][2], p=parts[0][3]) as ctx:
        d = torch.from_numpy(c0s[0]).cuda()
        with pytest.raises(esc.NonFiniteError):
            ctx.run_device(d.data_ptr(), 10, 0.01)
        torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy(), c0s[0])
