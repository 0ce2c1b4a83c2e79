"""The queued device-memory runs (esc_batch_run_device_async / esc_batch_wait and
esc_run_device_async / esc_wait): the same results as the blocking calls, the
outcome reported by the wait, and the misuse a queued run rules out.  Step counts
exercise the captured chunk graphs of 32, 16, 8, 4, 2 and 1 steps."""
import numpy as np
import pytest

import esc
from oracle import core_shell_oracle as orc

pytestmark = pytest.mark.gpu


def parts(sizes, seed0=70):
    return [orc.initial_fields(n, radius=0.3 * n, width=2.0, seed=seed0 + k) for k, n in enumerate(sizes)]


@pytest.mark.parametrize("steps", [0, 1, 7, 31, 63])
def test_batch_async_equals_blocking_and_oracle(steps):
    import torch
    ps = parts([32, 48, 32, 64])
    b = esc.Batch([p[1] for p in ps], precision="fp64")
    try:
        d1 = [torch.from_numpy(p[0]).cuda() for p in ps]
        d2 = [torch.from_numpy(p[0]).cuda() for p in ps]
        h1 = torch.zeros(len(ps) * (steps + 1) * 6, dtype=torch.float64, device="cuda")
        h2 = torch.zeros_like(h1)
        torch.cuda.synchronize()
        bad1 = b.run_device([x.data_ptr() for x in d1], steps, 0.01, h1.data_ptr())
        b.run_device_async([x.data_ptr() for x in d2], steps, 0.01, h2.data_ptr())
        bad2 = b.wait()
        assert bad1 == bad2 == [-1] * len(ps)
        for x, y in zip(d1, d2):
            assert torch.equal(x, y)
        assert torch.equal(h1, h2)
        for (c0, phi), x in zip(ps, d2):
            co, _ = orc.run_simulation(c0, phi, dt=0.01, steps=steps)
            assert np.max(np.abs(x.cpu().numpy() - co)) / np.max(np.abs(co)) < 1e-12
    finally:
        b.close()


def test_queued_run_must_be_waited_for():
    import torch
    ps = parts([32, 32])
    with esc.Batch([p[1] for p in ps], precision="fp64") as b:
        d = [torch.from_numpy(p[0]).cuda() for p in ps]
        torch.cuda.synchronize()
        with pytest.raises(esc.EscError) as ei:
            b.wait()                                        # nothing queued
        assert ei.value.status == esc.ESC_EINVAL
        b.run_device_async([x.data_ptr() for x in d], 5, 0.01)
        with pytest.raises(esc.EscError) as ei:
            b.run_device_async([x.data_ptr() for x in d], 5, 0.01)   # a second run before the wait
        assert ei.value.status == esc.ESC_EINVAL
        assert b.wait() == [-1, -1]
        assert b.run_device([x.data_ptr() for x in d], 3, 0.01) == [-1, -1]


def test_async_reports_nonfinite_in_the_wait():
    import torch
    ps = parts([32, 32])
    c_bad = ps[1][0].copy()
    c_bad[3, 3] = np.nan
    with esc.Batch([p[1] for p in ps], precision="fp64") as b:
        d = [torch.from_numpy(ps[0][0]).cuda(), torch.from_numpy(c_bad).cuda()]
        torch.cuda.synchronize()
        b.run_device_async([x.data_ptr() for x in d], 4, 0.01)
        assert b.wait() == [-1, 0]
        assert np.array_equal(np.isnan(d[1].cpu().numpy()), np.isnan(c_bad))   # c left as it was


def test_context_async_equals_blocking():
    import torch
    c0, phi = parts([64])[0]
    with esc.Context(phi) as ctx:
        d1 = torch.from_numpy(c0).cuda()
        d2 = torch.from_numpy(c0).cuda()
        torch.cuda.synchronize()
        ctx.run_device(d1.data_ptr(), 19, 0.01)
        ctx.run_device_async(d2.data_ptr(), 19, 0.01)
        ctx.wait()
        assert torch.equal(d1, d2)
