"""esc_run_noalloc: the allocation-free entry point, checked against esc_run.

Some callers may not allocate device memory (their GPU memory belongs to
another allocator or a fixed budget, or they cannot afford the device-wide
synchronisation of cudaMalloc/cudaFree inside their loop).  esc_run_noalloc
serves them: the caller passes device buffers for phi, c and the history, and
every intermediate lives in a fixed array inside the library.  This test
allocates its own device buffers with torch (the caller's side), calls the new
entry point through the C ABI twice in a row -- the second call reuses the
array the first one left behind -- and requires both results to match the
ordinary entry point to the FP64 tolerance of the other parity tests.  It lives
in its own file, collected last, and runs the same alone or after the suite.
"""
import ctypes

import numpy as np
import pytest

import esc
from esc import fields

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


def test_noalloc_matches_esc_run_on_two_calls():
    import torch

    n, steps, dt = 128, 60, 0.01
    p = esc.Parameters(P=6.0, chi=0.6)
    c0, phi = fields.initial_fields(n, radius=35.0, width=2.0, seed=11)
    with esc.Context(phi, p=p) as ctx:
        c_ref, h_ref = ctx.run(c0, dt=dt, steps=steps)

    fn = _entry()
    cp = esc._CParams.of(p)
    dphi = torch.from_numpy(phi).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        dc = torch.from_numpy(c0).cuda()
        dh = torch.full((6 * (steps + 1),), float("nan"), dtype=torch.float64, device="cuda")
        bad = ctypes.c_int64(123)
        st = fn(n, 1.0, dphi.data_ptr(), ctypes.byref(cp), dc.data_ptr(), steps, dt, dh.data_ptr(),
                ctypes.byref(bad), stream)
        assert st == 0, esc.load_library().esc_last_error(None).decode()
        assert bad.value == -1
        c = dc.cpu().numpy()
        h = dh.cpu().numpy().reshape(6, steps + 1).T
        assert _rel(c, c_ref) < RTOL_FP64, f"call {call}: c differs"
        for j in range(6):
            scale = max(np.max(np.abs(h_ref[:, j])), 1e-300)
            assert np.max(np.abs(h[:, j] - h_ref[:, j])) / scale < RTOL_FP64, f"call {call}: history column {j}"


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
