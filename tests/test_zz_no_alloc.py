"""esc_run_noalloc: the allocation-free entry point, checked against the oracle and esc_run.

Some callers may not allocate device memory (their GPU memory belongs to
another allocator or a fixed budget, or they cannot afford the device-wide
synchronisation of cudaMalloc/cudaFree inside their loop).  esc_run_noalloc
serves them: the caller passes device buffers for phi, c and the history, and
every intermediate lives in a fixed array inside the library.  These tests
allocate their own device buffers with torch (the caller's side) and call the
entry point through the C ABI twice in a row -- the second call reuses the array
the first one left behind -- at the smallest size with a factor of 3 (12), at
128 and at the limit (256, where the array is fully used).  Both results must
match the CPU oracle (core_shell.jl:84-103 restated) and the ordinary entry
point to the FP64 tolerance of the other parity tests.  A non-finite field must
give ESC_ENONFINITE with the step, like esc_run, and leave c unchanged.  The
file is collected last and runs the same alone or after the suite.
"""
import ctypes

import numpy as np
import pytest

import esc
from esc import fields
from oracle import core_shell_oracle as orc

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-12


def _entry():
    fn = esc.load_library().esc_run_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.POINTER(esc._CParams),
                   ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                   ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]
    return fn


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _call(fn, n, phi, p, c0, steps, dt):
    """One esc_run_noalloc call on torch-owned device buffers: (status, bad_step, c, history)."""
    import torch
    cp = esc._CParams.of(p)
    dphi = torch.from_numpy(phi).cuda()
    dc = torch.from_numpy(c0).cuda()
    dh = torch.full((6 * (steps + 1),), float("nan"), dtype=torch.float64, device="cuda")
    bad = ctypes.c_int64(123)
    stream = torch.cuda.current_stream().cuda_stream
    st = fn(n, 1.0, dphi.data_ptr(), ctypes.byref(cp), dc.data_ptr(), steps, dt, dh.data_ptr(),
            ctypes.byref(bad), stream)
    torch.cuda.synchronize()
    return st, bad.value, dc.cpu().numpy(), dh.cpu().numpy().reshape(6, steps + 1).T


def _hist_ok(h, ho):
    for j in range(6):
        scale = max(np.max(np.abs(ho[:, j])), 1e-300)
        if np.max(np.abs(h[:, j] - ho[:, j])) / scale >= RTOL_FP64:
            return False
    return True


@pytest.mark.parametrize("n,steps", [(12, 40), (128, 60), (256, 45)])
def test_noalloc_matches_oracle_and_esc_run_on_two_calls(n, steps):
    dt = 0.01
    p = esc.Parameters(P=6.0, chi=0.6)
    po = orc.Parameters(P=6.0, chi=0.6)
    c0, phi = fields.initial_fields(n, radius=0.27 * n, width=2.0, seed=11)
    co, ho = orc.run_simulation(c0, phi, dt=dt, steps=steps, p=po)
    with esc.Context(phi, p=p) as ctx:
        c_ref, h_ref = ctx.run(c0, dt=dt, steps=steps)
    fn = _entry()
    for call in range(2):
        st, bad, c, h = _call(fn, n, phi, p, c0, steps, dt)
        assert st == 0, esc.load_library().esc_last_error(None).decode()
        assert bad == -1
        assert _rel(c, co) < RTOL_FP64, f"call {call}: c differs from the oracle"
        assert _hist_ok(h, ho), f"call {call}: history differs from the oracle"
        assert _rel(c, c_ref) < RTOL_FP64, f"call {call}: c differs from esc_run"
        assert _hist_ok(h, h_ref), f"call {call}: history differs from esc_run"


def test_noalloc_nonfinite_like_esc_run():
    """A NaN in c0: ESC_ENONFINITE at step 0, c left as it was, the same as esc_run."""
    n, steps, dt = 64, 10, 0.01
    p = esc.Parameters()
    c0, phi = fields.initial_fields(n, radius=16.0)
    c0 = c0.copy()
    c0[5, 7] = np.nan
    fn = _entry()
    st, bad, c, h = _call(fn, n, phi, p, c0, steps, dt)
    assert st == esc.ESC_ENONFINITE
    assert bad == 0
    assert np.array_equal(np.isnan(c), np.isnan(c0)) and np.array_equal(c[~np.isnan(c)], c0[~np.isnan(c0)])
    with esc.Context(phi, p=p) as ctx:
        with pytest.raises(esc.NonFiniteError) as ei:
            ctx.run(c0, dt=dt, steps=steps)
    assert ei.value.step == bad
    # a run that blows up later: a huge step, same step index from both entry points
    c0, phi = fields.initial_fields(n, radius=16.0)
    st, bad, c, h = _call(fn, n, phi, p, c0, steps, 1e6)
    with esc.Context(phi, p=p) as ctx:
        try:
            ctx.run(c0, dt=1e6, steps=steps)
            ref_bad = -1
        except esc.NonFiniteError as e:
            ref_bad = e.step
    if ref_bad < 0:
        assert st == 0 and bad == -1
    else:
        assert st == esc.ESC_ENONFINITE and bad == ref_bad and bad >= 0
        assert np.array_equal(c, c0)


def test_noalloc_rejects_grids_above_its_limit():
    import torch

    fn = _entry()
    n = 512
    cp = esc._CParams.of(esc.Parameters())
    d = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    bad = ctypes.c_int64(0)
    st = fn(n, 1.0, d.data_ptr(), ctypes.byref(cp), d.data_ptr(), 1, 0.01, None, ctypes.byref(bad), None)
    assert st == esc.ESC_EINVAL
    assert "256" in esc.load_library().esc_last_error(None).decode()
