"""Coupled c-phi model in 3-D (ctypes over the esc_cphi_* functions of libesc.so).

The loop of the reference's 2023 3-D program (original/2023-3d/evolve.cu:74-186):
conserved composition c with mobility M = mobility h(phi) and an Allen-Cahn order
parameter phi, stepped by the stabilised semi-implicit Fourier update.  Fields are
C-ordered float64 arrays of shape (nx, ny, nz): element [i, j, k] sits at
k + nz*(j + ny*i), the reference's order.  All arithmetic runs in the library's
CUDA kernels; without the library every call raises.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Tuple

import numpy as np

from . import (ESC_EMASS, ESC_ENONFINITE, ESC_OK, EscError, NonFiniteError, _CCphiParams, _dp, _ptr, _vp,
               load_library)

COMPLETED, CONVERGED, OUT_OF_BOUNDS, MASS_ERROR, NONFINITE = range(5)
COMPERR = 1.0e-8  # binary.h:14 of the reference's 3-D program

__all__ = ["CoupledParameters", "Coupled", "MassError", "run_coupled", "supported_axis",
           "COMPLETED", "CONVERGED", "OUT_OF_BOUNDS", "MASS_ERROR", "NONFINITE"]


@dataclasses.dataclass(frozen=True)
class CoupledParameters:
    """Constants of original/2023-3d/InputParams:13-22."""

    A: float = 2.0
    B: float = 1.0
    chi: float = 0.5
    P: float = 6.0
    ca: float = 0.5
    cb1: float = 0.0
    cb2: float = 1.0
    A0: float = 0.08
    kappa_c: float = 2.0
    kappa_phi: float = 10.0
    mobility: float = 1.0
    relax: float = 0.001
    Q: float = 0.5

    def c_struct(self) -> _CCphiParams:
        return _CCphiParams(*[float(getattr(self, f)) for f, _ in _CCphiParams._fields_])


class MassError(EscError):
    """The mean composition moved by more than comperr in one step
    ("Elements NOT conserved", original/2023-3d/evolve.cu:149-154)."""

    def __init__(self, step: int, message: str):
        super().__init__(ESC_EMASS, message)
        self.step = int(step)


def supported_axis(n: int) -> bool:
    return bool(load_library().esc_cphi_supported_size(int(n)))


class Coupled:
    """A coupled-model context for one grid (esc_cphi_create)."""

    def __init__(self, shape: Tuple[int, int, int], spacing=(1.0, 1.0, 1.0),
                 params: CoupledParameters = CoupledParameters()):
        lib = load_library()
        self.shape = tuple(int(v) for v in shape)
        self._h = _vp()
        cp = params.c_struct()
        st = lib.esc_cphi_create(ctypes.byref(self._h), *self.shape, *[float(v) for v in spacing],
                                 ctypes.byref(cp))
        if st != ESC_OK:
            raise EscError(st, lib.esc_last_error(None).decode())

    def _err(self) -> str:
        return load_library().esc_cphi_last_error(self._h).decode()

    def _check(self, st: int, done: int):
        if st == ESC_ENONFINITE:
            raise NonFiniteError(done, self._err())
        if st == ESC_EMASS:
            raise MassError(done, self._err())
        if st != ESC_OK:
            raise EscError(st, self._err())

    def run(self, c0, phi0, dt: float = 0.01, steps: int = 100, tolerance: float = 0.0,
            comperr: float = COMPERR):
        """Returns (c, phi, history, steps_done, stop_reason); history has shape (steps+1, 6)
        with rows [s*dt, mean c, mean phi, min c, max c, max|c_s - c_(s-1)|]."""
        c = np.array(c0, dtype=np.float64, order="C", copy=True)
        phi = np.array(phi0, dtype=np.float64, order="C", copy=True)
        if c.shape != self.shape or phi.shape != self.shape:
            raise ValueError(f"fields must have shape {self.shape}")
        hist = np.zeros((6, steps + 1))
        done = ctypes.c_int64(-1)
        reason = ctypes.c_int(-1)
        st = load_library().esc_cphi_run(self._h, _ptr(c), _ptr(phi), int(steps), float(dt), float(tolerance),
                                         float(comperr), _ptr(hist), ctypes.byref(done), ctypes.byref(reason))
        self._check(st, done.value)
        return c, phi, hist.T.copy(), int(done.value), int(reason.value)

    def run_device(self, c_ptr: int, phi_ptr: int, steps: int, dt: float, tolerance: float = 0.0,
                   comperr: float = COMPERR, hist_ptr: int = 0):
        """esc_cphi_run_device on caller-owned device arrays; returns (steps_done, stop_reason)."""
        done = ctypes.c_int64(-1)
        reason = ctypes.c_int(-1)
        st = load_library().esc_cphi_run_device(self._h, _vp(c_ptr), _vp(phi_ptr), int(steps), float(dt),
                                                float(tolerance), float(comperr),
                                                _vp(hist_ptr) if hist_ptr else None, ctypes.byref(done),
                                                ctypes.byref(reason))
        self._check(st, done.value)
        return int(done.value), int(reason.value)

    KERNELS = ("z fwd local", "y fwd x2", "x mu/phi", "y inv", "z inv mu + z stencil", "y stencil",
               "x stencil", "z fwd div", "y fwd", "x c update", "y inv x2", "z inv final")

    def profile(self, steps: int = 5):
        """Mean time (ms) of each of the twelve stages of a step (esc_cphi_profile),
        stepping on from the fields of the last run."""
        ms = np.zeros(12)
        st = load_library().esc_cphi_profile(self._h, int(steps), _ptr(ms))
        if st != ESC_OK:
            raise EscError(st, self._err())
        return dict(zip(self.KERNELS, ms.tolist()))

    def set_stream(self, stream_ptr: int) -> None:
        st = load_library().esc_cphi_set_stream(self._h, _vp(stream_ptr) if stream_ptr else None)
        if st != ESC_OK:
            raise EscError(st, self._err())

    def close(self) -> None:
        if self._h:
            load_library().esc_cphi_destroy(self._h)
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


def run_coupled(c0, phi0, dt: float = 0.01, steps: int = 100, spacing=(1.0, 1.0, 1.0),
                params: CoupledParameters = CoupledParameters(), tolerance: float = 0.0, comperr: float = COMPERR):
    """One-shot run of the coupled model: (c, phi, history, steps_done, stop_reason)."""
    with Coupled(np.shape(c0), spacing, params) as ctx:
        return ctx.run(c0, phi0, dt, steps, tolerance, comperr)


def initial_fields(nx: int, ny: int, nz: int, radius: float, c_mean: float = 0.5, noise: float = 0.05,
                   seed: int = 2938, params: CoupledParameters = CoupledParameters(), phicutoff: float = 0.5):
    """Sharp spherical particle and noisy composition of original/2023-3d/init_conf.cu:55-125
    (flag 1): phi = 1 for r < radius about (nx/2, ny/2, nz/2), else 0; inside
    (phi > phicutoff) c = c_mean (cb1 + cb2) + u - <u>, u uniform in [-noise, noise) with its
    particle mean removed; outside c = ca.  u comes from NumPy's PCG64 seeded with `seed`
    (the reference draws it with cuRAND)."""
    i = np.arange(nx)[:, None, None] - nx // 2
    j = np.arange(ny)[None, :, None] - ny // 2
    k = np.arange(nz)[None, None, :] - nz // 2
    r = np.sqrt((i * i + j * j + k * k).astype(np.float64))
    phi = np.where(r < radius, 1.0, 0.0)
    u = (2.0 * np.random.default_rng(seed).random((nx, ny, nz)) - 1.0) * noise
    inside = phi > phicutoff
    mean = u[inside].mean() if inside.any() else 0.0
    c = np.where(inside, c_mean * (params.cb1 + params.cb2) + u - mean, params.ca)
    return c, phi
