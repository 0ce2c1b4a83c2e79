"""The C-ABI library on a machine without a GPU: it loads, exports every
function include/esc.h declares, and validates arguments before touching CUDA.
No compute call is made here."""
import ctypes
import os
import re

import numpy as np
import pytest

import esc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "esc.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(esc_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("esc_create", "esc_run", "esc_run_device", "esc_destroy", "esc_last_error",
                     "esc_batch_create", "esc_batch_run", "esc_batch_destroy", "esc_run_noalloc"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = esc.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} declared in include/esc.h but not exported"


def test_binding_covers_every_declared_symbol():
    bound = {name for name, _, _ in esc._SIGNATURES} | {"esc_run_noalloc"}
    assert set(declared_functions()) <= bound


def test_default_params_match_reference():
    lib = esc.load_library()
    cp = esc._CParams()
    lib.esc_default_params(ctypes.byref(cp))
    got = tuple(getattr(cp, f) for f, _ in esc._CParams._fields_)
    p = esc.Parameters()
    assert got == (p.A, p.B, p.chi, p.P, p.ca, p.cb, p.cc, p.kappa, p.mobility, p.Q)
    assert got == (2.0, 4.0, 0.5, 5.0, 0.5, 0.0, 1.0, 2.0, 1.0, 0.5)   # core_shell.jl:4-15


def test_supported_sizes():
    # tuned kernel sets
    ok = [8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536, 2048, 3072, 4096]
    # runtime-size kernels: any n in [2, 4096] with prime factors <= 127, or any n <= 512 (odd, prime, radix 5, 7)
    ok += [2, 3, 4, 6, 10, 15, 65, 97, 100, 101, 130, 160, 255, 320, 509, 1000, 2187, 4095]
    for n in ok:
        assert esc.supported_size(n), n
    for n in (0, 1, -8, 4097, 8192, 521, 1009, 4093, 2 * 257 * 3):
        assert not esc.supported_size(n), n
    assert b"sm_100a" in esc.load_library().esc_version()


def test_invalid_arguments_rejected_before_cuda():
    lib = esc.load_library()
    cp = esc._CParams.of(esc.Parameters())
    h = ctypes.c_void_p()
    phi = np.zeros((1009, 1009))
    st = lib.esc_create(ctypes.byref(h), 1009, 1.0, phi.ctypes.data_as(esc._dp), ctypes.byref(cp), 0)
    assert st == esc.ESC_EINVAL and not h.value
    assert b"unsupported grid size 1009" in lib.esc_last_error(None)
    st = lib.esc_create(ctypes.byref(h), 64, 1.0, None, ctypes.byref(cp), 0)
    assert st == esc.ESC_EINVAL
    phi = np.zeros((64, 64))
    st = lib.esc_create(ctypes.byref(h), 64, -1.0, phi.ctypes.data_as(esc._dp), ctypes.byref(cp), 0)
    assert st == esc.ESC_EINVAL
    bad = esc._CParams.of(esc.Parameters(P=float("nan")))
    st = lib.esc_create(ctypes.byref(h), 64, 1.0, phi.ctypes.data_as(esc._dp), ctypes.byref(bad), 0)
    assert st == esc.ESC_EINVAL
    st = lib.esc_create(ctypes.byref(h), 64, 1.0, phi.ctypes.data_as(esc._dp), ctypes.byref(cp), 7)
    assert st == esc.ESC_EINVAL
    assert lib.esc_run(None, None, 1, 0.01, None, None) == esc.ESC_EINVAL
    assert lib.esc_batch_run(None, None, 1, 0.01, None, None) == esc.ESC_EINVAL
    lib.esc_destroy(None)
    lib.esc_batch_destroy(None)


def test_noalloc_size_limit_checked_before_cuda():
    lib = esc.load_library()
    fn = lib.esc_run_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.POINTER(esc._CParams),
                   ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                   ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]
    cp = esc._CParams.of(esc.Parameters())
    bad = ctypes.c_int64(0)
    assert fn(512, 1.0, 1, ctypes.byref(cp), 1, 1, 0.01, None, ctypes.byref(bad), None) == esc.ESC_EINVAL
    assert bad.value == -1
    assert fn(100, 1.0, 1, ctypes.byref(cp), 1, 1, 0.01, None, ctypes.byref(bad), None) == esc.ESC_EINVAL


def test_no_gpu_fails_loudly_not_silently():
    from conftest import HAS_GPU
    if HAS_GPU:
        pytest.skip("a GPU is present")
    with pytest.raises(esc.EscError) as ei:
        esc.Context(np.zeros((64, 64)))
    assert ei.value.status in (esc.ESC_ECUDA, esc.ESC_ENOMEM)


def test_concurrent_creations_fail_independently():
    """Creations from many host threads at once (they are serialised inside the
    library): every call returns, the lock is released on each error path, and
    each thread reads its own message from esc_last_error(NULL).  All of them fail
    argument validation, so no CUDA call is made."""
    import threading
    lib = esc.load_library()
    cp = esc._CParams.of(esc.Parameters())
    results = {}

    def attempt(i):
        h = ctypes.c_void_p()
        n = (521, 523, 541, 547, 557, 563, 569, 571)[i]   # primes above 512: no kernels for these sizes
        phi = np.zeros((n, n))
        for _ in range(50):
            st = lib.esc_create(ctypes.byref(h), n, 1.0, phi.ctypes.data_as(esc._dp), ctypes.byref(cp), 0)
            msg = lib.esc_last_error(None)
            if st != esc.ESC_EINVAL or h.value or f"unsupported grid size {n}".encode() not in msg:
                results[i] = (st, h.value, msg)
                return
        results[i] = "ok"

    threads = [threading.Thread(target=attempt, args=(i,)) for i in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=60)
    assert not any(t.is_alive() for t in threads)
    assert results == {i: "ok" for i in range(8)}
