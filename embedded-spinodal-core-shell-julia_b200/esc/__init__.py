"""Python host side of the B200 Cahn-Hilliard stepper (ctypes over libesc.so).

Mirrors the driver of the reference Julia model
(saswataiith/embedded-spinodal-core-shell-julia, ``core_shell.jl``):

* :class:`Parameters` is field-for-field ``Parameters`` (core_shell.jl:4-15);
* :func:`run_simulation` has the signature and results of
  ``run_simulation(c0, phi; dt, steps, spacing, p)`` (core_shell.jl:84-103):
  it returns ``(c, history)`` with ``history`` of shape ``(steps+1, 6)`` and
  rows ``[s*dt, mean c, energy, min c, max c, dissipation]``, and raises
  :class:`NonFiniteError` (``"Non-finite composition at step s"``, as
  core_shell.jl:93) when the composition stops being finite.

All numerical work runs in the CUDA kernels of ``libesc.so``; this module only
moves arrays across the C ABI declared in ``include/esc.h``.  There is no CPU
path: when the library or a GPU is missing every call raises.

Array layout: a field is a C-ordered ``float64`` NumPy array ``a[y, x]`` of
shape ``(n, n)`` -- byte-for-byte the column-major Julia ``Matrix{Float64}``
whose first index is x.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
from typing import Optional, Sequence

import numpy as np

__all__ = [
    "Parameters", "NonFiniteError", "EscError", "Context", "Batch", "run_simulation",
    "supported_size", "load_library", "FP64", "MIXED", "library_path",
]

FP64 = 0
MIXED = 1
_PREC = {"fp64": FP64, "mixed": MIXED, FP64: FP64, MIXED: MIXED}

ESC_OK, ESC_EINVAL, ESC_ECUDA, ESC_ENONFINITE, ESC_ETIMEOUT, ESC_ENOMEM, ESC_EMASS = range(7)
_STATUS_NAMES = {0: "ESC_OK", 1: "ESC_EINVAL", 2: "ESC_ECUDA", 3: "ESC_ENONFINITE",
                 4: "ESC_ETIMEOUT", 5: "ESC_ENOMEM", 6: "ESC_EMASS"}


@dataclasses.dataclass(frozen=True)
class Parameters:
    """Model constants with the defaults of core_shell.jl:4-15."""

    A: float = 2.0
    B: float = 4.0
    chi: float = 0.5
    P: float = 5.0
    ca: float = 0.5
    cb: float = 0.0
    cc: float = 1.0
    kappa: float = 2.0
    mobility: float = 1.0
    Q: float = 0.5


class EscError(RuntimeError):
    """A failed library call; ``status`` is the esc_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class NonFiniteError(EscError):
    """``error("Non-finite composition at step $s")`` of core_shell.jl:93."""

    def __init__(self, step: int, message: str = ""):
        super().__init__(ESC_ENONFINITE, message or f"Non-finite composition at step {step}")
        self.step = int(step)


class _CParams(ctypes.Structure):
    _fields_ = [(f, ctypes.c_double) for f in
                ("A", "B", "chi", "P", "ca", "cb", "cc", "kappa", "mobility", "Q")]

    @classmethod
    def of(cls, p: Parameters) -> "_CParams":
        return cls(*[float(getattr(p, f)) for f, _ in cls._fields_])


class _CCphiParams(ctypes.Structure):
    """esc_cphi_params: constants of the coupled c-phi model (original/2023-3d/InputParams:13-22)."""
    _fields_ = [(f, ctypes.c_double) for f in
                ("A", "B", "chi", "P", "ca", "cb1", "cb2", "A0", "kappa_c", "kappa_phi", "mobility", "relax", "Q")]


_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p

# (name, restype, argtypes) for every function of include/esc.h
_SIGNATURES = [
    ("esc_default_params", None, [ctypes.POINTER(_CParams)]),
    ("esc_supported_size", ctypes.c_int, [ctypes.c_int]),
    ("esc_version", ctypes.c_char_p, []),
    ("esc_create", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_double, _dp,
                                  ctypes.POINTER(_CParams), ctypes.c_int]),
    ("esc_run", ctypes.c_int, [_vp, _dp, ctypes.c_int, ctypes.c_double, _dp, _i64p]),
    ("esc_run_device", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_double, _vp, _i64p]),
    ("esc_set_stream", ctypes.c_int, [_vp, _vp]),
    ("esc_run_device_async", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_double, _vp]),
    ("esc_wait", ctypes.c_int, [_vp, _i64p]),
    ("esc_last_error", ctypes.c_char_p, [_vp]),
    ("esc_uses_cluster", ctypes.c_int, [_vp]),
    ("esc_destroy", None, [_vp]),
    ("esc_adjoint", ctypes.c_int, [_vp, _dp, ctypes.c_int, ctypes.c_double, _dp, ctypes.c_double, ctypes.c_int,
                                   _dp, _dp, _dp]),
    ("esc_batch_create", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                        _dp, ctypes.POINTER(_dp), ctypes.POINTER(_CParams), ctypes.c_int]),
    ("esc_batch_run", ctypes.c_int, [_vp, ctypes.POINTER(_dp), ctypes.c_int, ctypes.c_double,
                                     ctypes.POINTER(_dp), _i64p]),
    ("esc_batch_run_device", ctypes.c_int, [_vp, ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_double,
                                            _vp, _i64p]),
    ("esc_batch_set_stream", ctypes.c_int, [_vp, _vp]),
    ("esc_batch_run_device_async", ctypes.c_int, [_vp, ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_double, _vp]),
    ("esc_batch_wait", ctypes.c_int, [_vp, _i64p]),
    ("esc_batch_adjoint", ctypes.c_int, [_vp, ctypes.POINTER(_dp), ctypes.c_int, ctypes.c_double,
                                         ctypes.POINTER(_dp), ctypes.c_double, ctypes.c_int, ctypes.POINTER(_dp),
                                         _dp, _dp]),
    ("esc_batch_profile_phases", ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                                _dp]),
    ("esc_batch_describe", ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_int]),
    ("esc_particle_device", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, ctypes.c_double,
                                           _vp, _vp]),
    ("esc_noise_device", ctypes.c_int, [ctypes.c_int, _vp, ctypes.c_double, ctypes.c_double, ctypes.c_uint64,
                                        _vp, _vp]),
    ("esc_julia_rand", ctypes.c_int, [ctypes.c_uint64, _dp, ctypes.c_int64]),
    ("esc_batch_last_error", ctypes.c_char_p, [_vp]),
    ("esc_batch_destroy", None, [_vp]),
    ("esc_cphi_default_params", None, [ctypes.POINTER(_CCphiParams)]),
    ("esc_cphi_supported_size", ctypes.c_int, [ctypes.c_int]),
    ("esc_cphi_create", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.POINTER(_CCphiParams)]),
    ("esc_cphi_run", ctypes.c_int, [_vp, _dp, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    _dp, _i64p, ctypes.POINTER(ctypes.c_int)]),
    ("esc_cphi_run_device", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, _vp, _i64p, ctypes.POINTER(ctypes.c_int)]),
    ("esc_cphi_set_stream", ctypes.c_int, [_vp, _vp]),
    ("esc_cphi_profile", ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    ("esc_cphi_last_error", ctypes.c_char_p, [_vp]),
    ("esc_cphi_destroy", None, [_vp]),
]

_LIB: Optional[ctypes.CDLL] = None


def library_path() -> str:
    """Path of libesc.so: $ESC_LIBRARY if set, else next to this file."""
    return os.environ.get("ESC_LIBRARY") or os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                         "libesc.so")


def load_library() -> ctypes.CDLL:
    """Loads libesc.so (once) and declares the C signatures.  Raises OSError
    when the library has not been built; there is no substitute."""
    global _LIB
    if _LIB is None:
        path = library_path()
        if not os.path.exists(path):
            raise OSError(f"libesc.so not found at {path}; build it with "
                          "`make -C embedded-spinodal-core-shell-julia_b200/csrc`")
        lib = ctypes.CDLL(path)
        for name, res, args in _SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


SHAPES = {"disc": 0, "band": 1, "ellipse": 2, "annulus": 3, "squircle": 4, "elliptic_shell": 5, "elliptic_hole": 6}


def particle_device(shape: str, n: int, phi_ptr: int, params, width: float = 2.0, spacing: float = 1.0,
                    stream_ptr: int = 0) -> None:
    """Fills the device array at `phi_ptr` (n*n doubles) with a particle shape
    (esc_particle_device; shapes and parameters as in include/esc.h)."""
    q = np.zeros(4)
    q[:len(params)] = params
    st = load_library().esc_particle_device(SHAPES[shape], int(n), float(spacing), _ptr(q), float(width),
                                            _vp(phi_ptr), _vp(stream_ptr) if stream_ptr else None)
    if st != ESC_OK:
        _raise(st, load_library().esc_last_error(None).decode())


def noise_device(n: int, c_ptr: int, seed: int, phi_ptr: int = 0, mean: float = 0.5, amplitude: float = 0.01,
                 stream_ptr: int = 0) -> None:
    """Fills the device array at `c_ptr` with counter-based noise (esc_noise_device):
    inside the particle at `phi_ptr` with its interior mean removed, or over the whole
    field when phi_ptr is 0."""
    st = load_library().esc_noise_device(int(n), _vp(phi_ptr) if phi_ptr else None, float(mean), float(amplitude),
                                         ctypes.c_uint64(int(seed) & 0xFFFFFFFFFFFFFFFF), _vp(c_ptr),
                                         _vp(stream_ptr) if stream_ptr else None)
    if st != ESC_OK:
        _raise(st, load_library().esc_last_error(None).decode())


def supported_size(n: int) -> bool:
    return bool(load_library().esc_supported_size(int(n)))


def _field(a, n: int, name: str) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.shape != (n, n):
        raise ValueError(f"{name} must have shape ({n}, {n}), got {a.shape}")
    return a


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _raise(status: int, msg: str, bad_step: int = -1):
    if status == ESC_ENONFINITE:
        raise NonFiniteError(bad_step, msg)
    raise EscError(status, msg)


class Context:
    """One particle on one GPU (wraps esc_create / esc_run / esc_destroy)."""

    def __init__(self, phi, spacing: float = 1.0, p: Parameters = Parameters(), precision="fp64"):
        lib = load_library()
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        if phi.ndim != 2 or phi.shape[0] != phi.shape[1]:
            raise ValueError(f"phi must be square, got shape {phi.shape}")
        self.n = int(phi.shape[0])
        self.precision = _PREC[precision]
        self._h = _vp()
        cp = _CParams.of(p)
        st = lib.esc_create(ctypes.byref(self._h), self.n, float(spacing), _ptr(phi), ctypes.byref(cp),
                            self.precision)
        if st != ESC_OK:
            _raise(st, lib.esc_last_error(None).decode())

    def _err(self) -> str:
        return load_library().esc_last_error(self._h).decode()

    def run(self, c0, dt: float = 0.01, steps: int = 1000, with_history: bool = True):
        """Returns ``(c, history)`` after ``steps`` steps (history None if not asked)."""
        c = _field(c0, self.n, "c0").copy()
        hist = np.zeros((6, steps + 1)) if with_history else None  # column-major (steps+1) x 6
        bad = ctypes.c_int64(-1)
        st = load_library().esc_run(self._h, _ptr(c), int(steps), float(dt),
                                    _ptr(hist) if hist is not None else None, ctypes.byref(bad))
        if st != ESC_OK:
            _raise(st, self._err(), bad.value)
        return c, (hist.T.copy() if hist is not None else None)

    def adjoint(self, c0, c_target, dt: float = 0.01, steps: int = 100, lambda_F: float = 1e-3,
                ckpt_every: int = 0):
        """(L, dL/dc0, dL/d(P, chi, kappa, M0)) for L = 1/2 |c_T - c_target|^2 + lambda_F F[c_T]."""
        c0 = _field(c0, self.n, "c0")
        ct = _field(c_target, self.n, "c_target")
        g = np.zeros((self.n, self.n))
        dp = np.zeros(4)
        L = ctypes.c_double(0.0)
        st = load_library().esc_adjoint(self._h, _ptr(c0), int(steps), float(dt), _ptr(ct), float(lambda_F),
                                        int(ckpt_every), _ptr(g), _ptr(dp), ctypes.byref(L))
        if st != ESC_OK:
            _raise(st, self._err())
        return L.value, g, dp

    def run_device(self, c_ptr: int, steps: int, dt: float, hist_ptr: int = 0) -> None:
        """esc_run_device on caller-owned device buffers (raw addresses)."""
        bad = ctypes.c_int64(-1)
        st = load_library().esc_run_device(self._h, _vp(c_ptr), int(steps), float(dt),
                                           _vp(hist_ptr) if hist_ptr else None, ctypes.byref(bad))
        if st != ESC_OK:
            _raise(st, self._err(), bad.value)

    def run_device_async(self, c_ptr: int, steps: int, dt: float, hist_ptr: int = 0) -> None:
        """esc_run_device_async: queues the run on the context's stream and returns; call wait()."""
        st = load_library().esc_run_device_async(self._h, _vp(c_ptr), int(steps), float(dt),
                                                 _vp(hist_ptr) if hist_ptr else None)
        if st != ESC_OK:
            _raise(st, self._err())

    def wait(self) -> None:
        """esc_wait: waits for the queued run; raises NonFiniteError like run_device."""
        bad = ctypes.c_int64(-1)
        st = load_library().esc_wait(self._h, ctypes.byref(bad))
        if st != ESC_OK:
            _raise(st, self._err(), bad.value)

    @property
    def uses_cluster(self) -> bool:
        """True when this context's runs go through the cluster-resident kernel (esc_uses_cluster)."""
        return bool(load_library().esc_uses_cluster(self._h))

    def set_stream(self, stream_ptr: int) -> None:
        st = load_library().esc_set_stream(self._h, _vp(stream_ptr) if stream_ptr else None)
        if st != ESC_OK:
            _raise(st, self._err())

    def close(self) -> None:
        if self._h:
            load_library().esc_destroy(self._h)
            self._h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """An ensemble of independent particles (sizes may differ) advanced together."""

    def __init__(self, phis: Sequence, spacings=None, params=None, precision="mixed"):
        lib = load_library()
        self.phis = [np.ascontiguousarray(f, dtype=np.float64) for f in phis]
        self.count = len(self.phis)
        if self.count < 1:
            raise ValueError("a batch needs at least one particle")
        self.n = [int(f.shape[0]) for f in self.phis]
        for f in self.phis:
            if f.ndim != 2 or f.shape[0] != f.shape[1]:
                raise ValueError(f"phi must be square, got shape {f.shape}")
        spacings = [1.0] * self.count if spacings is None else [float(s) for s in spacings]
        params = [Parameters()] * self.count if params is None else list(params)
        if len(spacings) != self.count or len(params) != self.count:
            raise ValueError("spacings/params must have one entry per particle")
        self.precision = _PREC[precision]
        narr = (ctypes.c_int * self.count)(*self.n)
        dxarr = (ctypes.c_double * self.count)(*spacings)
        parr = (_dp * self.count)(*[_ptr(f) for f in self.phis])
        cps = (_CParams * self.count)(*[_CParams.of(p) for p in params])
        self._h = _vp()
        st = lib.esc_batch_create(ctypes.byref(self._h), self.count, narr, dxarr, parr, cps, self.precision)
        if st != ESC_OK:
            _raise(st, lib.esc_batch_last_error(None).decode())

    def _err(self) -> str:
        return load_library().esc_batch_last_error(self._h).decode()

    def run(self, c0s: Sequence, dt: float = 0.01, steps: int = 1000, with_history: bool = True):
        """Returns ``(cs, histories, bad_steps)``; ``bad_steps[i]`` is -1 or the
        step at which particle i became non-finite (its c is then not updated)."""
        if len(c0s) != self.count:
            raise ValueError("one initial field per particle")
        cs = [_field(c, n, "c0").copy() for c, n in zip(c0s, self.n)]
        hs = [np.zeros((6, steps + 1)) for _ in cs] if with_history else None
        carr = (_dp * self.count)(*[_ptr(c) for c in cs])
        harr = (_dp * self.count)(*[_ptr(h) for h in hs]) if hs is not None else None
        bad = (ctypes.c_int64 * self.count)()
        st = load_library().esc_batch_run(self._h, carr, int(steps), float(dt), harr, bad)
        bads = [int(b) for b in bad]
        if st not in (ESC_OK, ESC_ENONFINITE):
            _raise(st, self._err())
        return cs, ([h.T.copy() for h in hs] if hs is not None else None), bads

    def run_device(self, c_ptrs: Sequence[int], steps: int, dt: float, hist_ptr: int = 0):
        carr = (_vp * self.count)(*[_vp(p) for p in c_ptrs])
        bad = (ctypes.c_int64 * self.count)()
        st = load_library().esc_batch_run_device(self._h, carr, int(steps), float(dt),
                                                 _vp(hist_ptr) if hist_ptr else None, bad)
        if st not in (ESC_OK, ESC_ENONFINITE):
            _raise(st, self._err())
        return [int(b) for b in bad]

    def run_device_async(self, c_ptrs: Sequence[int], steps: int, dt: float, hist_ptr: int = 0) -> None:
        """esc_batch_run_device_async: queues the run on the batch's stream and returns; call wait()."""
        carr = (_vp * self.count)(*[_vp(p) for p in c_ptrs])
        st = load_library().esc_batch_run_device_async(self._h, carr, int(steps), float(dt),
                                                       _vp(hist_ptr) if hist_ptr else None)
        if st != ESC_OK:
            _raise(st, self._err())

    def wait(self):
        """esc_batch_wait: waits for the queued run; returns the per-instance bad steps like run_device."""
        bad = (ctypes.c_int64 * self.count)()
        st = load_library().esc_batch_wait(self._h, bad)
        if st not in (ESC_OK, ESC_ENONFINITE):
            _raise(st, self._err())
        return [int(b) for b in bad]

    def profile_phases(self, steps: int = 5):
        """Mean kernel time (ms) of each phase per size group on the current
        device state: list of (n, count, [row_a, col_a, row_b, col_b])."""
        lib = load_library()
        ng = ctypes.c_int(0)
        st = lib.esc_batch_profile_phases(self._h, int(steps), ctypes.byref(ng), None, None, None)
        if st != ESC_OK:
            _raise(st, self._err())
        gn = (ctypes.c_int * ng.value)()
        gc = (ctypes.c_int * ng.value)()
        ms = np.zeros(4 * ng.value)
        st = lib.esc_batch_profile_phases(self._h, int(steps), ctypes.byref(ng), gn, gc, _ptr(ms))
        if st != ESC_OK:
            _raise(st, self._err())
        return [(int(gn[i]), int(gc[i]), [float(x) for x in ms[4 * i:4 * i + 4]]) for i in range(ng.value)]

    def adjoint(self, c0s: Sequence, c_targets: Sequence, dt: float = 0.01, steps: int = 100,
                lambda_F: float = 1e-3, ckpt_every: int = 0, with_field_gradients: bool = True):
        """Per particle (L, dL/dc0, dL/d(P, chi, kappa, M0)) for
        L = 1/2 |c_T - c_target|^2 + lambda_F F[c_T]; all particles must share one grid size.
        Returns (L array (count,), list of dL/dc0 fields or None, (count, 4) array)."""
        if len(c0s) != self.count or len(c_targets) != self.count:
            raise ValueError("one initial field and one target per particle")
        cs = [_field(c, n, "c0") for c, n in zip(c0s, self.n)]
        ts = [_field(c, n, "c_target") for c, n in zip(c_targets, self.n)]
        gs = [np.zeros((n, n)) for n in self.n] if with_field_gradients else None
        dp = np.zeros((self.count, 4))
        L = np.zeros(self.count)
        carr = (_dp * self.count)(*[_ptr(c) for c in cs])
        tarr = (_dp * self.count)(*[_ptr(c) for c in ts])
        garr = (_dp * self.count)(*[_ptr(x) for x in gs]) if gs is not None else None
        st = load_library().esc_batch_adjoint(self._h, carr, int(steps), float(dt), tarr, float(lambda_F),
                                              int(ckpt_every), garr, _ptr(dp), _ptr(L))
        if st != ESC_OK:
            _raise(st, self._err())
        return L, gs, dp

    def describe(self):
        """The autotuner's choice of kernel families per size group (list of dicts)."""
        import json
        lib = load_library()
        need = lib.esc_batch_describe(self._h, None, 0)
        buf = ctypes.create_string_buffer(max(need, 1))
        lib.esc_batch_describe(self._h, buf, len(buf))
        return json.loads(buf.value.decode())

    def set_stream(self, stream_ptr: int) -> None:
        st = load_library().esc_batch_set_stream(self._h, _vp(stream_ptr) if stream_ptr else None)
        if st != ESC_OK:
            _raise(st, self._err())

    def close(self) -> None:
        if self._h:
            load_library().esc_batch_destroy(self._h)
            self._h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_simulation(c0, phi, dt: float = 0.01, steps: int = 1000, spacing: float = 1.0,
                   p: Parameters = Parameters(), precision="fp64"):
    """Drop-in for ``run_simulation`` of core_shell.jl:84-103 (without the CSV
    output, which stays with the caller).  Returns ``(c, history)``."""
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    with Context(phi, spacing=spacing, p=p, precision=precision) as ctx:
        return ctx.run(c0, dt=dt, steps=steps)
