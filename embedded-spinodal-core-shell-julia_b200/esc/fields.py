"""Host-side generators of particle fields and initial compositions.

These build the inputs of a run: the tanh disc and initial composition of
``initial_fields`` (reference core_shell.jl:27-37), an elliptical particle, and
whole-field noise for ensembles.  Noise is the reference's own stream:
``rand(MersenneTwister(seed), n, n)`` (core_shell.jl:32), reproduced bit for bit
by the library's host function ``esc_julia_rand`` (Julia 1.12's seed hashing and
dSFMT-19937), so ``initial_fields(n; radius, width, seed)`` returns exactly the
reference's inputs.  Arrays are C-ordered ``a[y, x]`` (the bytes of the
column-major Julia matrix).
"""
from __future__ import annotations

import numpy as np

__all__ = ["particle_disc", "particle_ellipse", "julia_rand", "interior_noise", "whole_field_noise",
           "initial_fields"]


def julia_rand(seed: int, n: int, m: int | None = None) -> np.ndarray:
    """``rand(MersenneTwister(seed), n, m)`` as a C-ordered array ``a[j, i]`` (esc_julia_rand)."""
    from . import _ptr, _raise, load_library
    m = n if m is None else m
    out = np.empty((m, n), dtype=np.float64)
    lib = load_library()
    st = lib.esc_julia_rand(int(seed) & 0xFFFFFFFFFFFFFFFF, _ptr(out), out.size)
    if st != 0:
        _raise(st, "esc_julia_rand: bad arguments")
    return out


def _centred(n: int, spacing: float) -> np.ndarray:
    # x = (i - 1 - n÷2) * spacing for Julia's 1-based i  (core_shell.jl:29)
    return (np.arange(n) - n // 2) * spacing


def particle_disc(n: int, spacing: float = 1.0, radius: float = 70.0, width: float = 4.0) -> np.ndarray:
    """phi = 0.5 (1 - tanh((r - radius) / width)), centred on index n÷2 (core_shell.jl:29-30)."""
    x = _centred(n, spacing)
    r = np.hypot(x.reshape(1, n), x.reshape(n, 1))
    return 0.5 * (1.0 - np.tanh((r - radius) / width))


def particle_ellipse(n: int, a: float, b: float, width: float, spacing: float = 1.0) -> np.ndarray:
    """phi = 0.5 (1 - tanh((sqrt((x b/a)^2 + y^2) - b) / width)); semi-axis a along x, b along y."""
    x = _centred(n, spacing).reshape(1, n)
    y = _centred(n, spacing).reshape(n, 1)
    return 0.5 * (1.0 - np.tanh((np.sqrt((x * b / a) ** 2 + y ** 2) - b) / width))


def interior_noise(phi: np.ndarray, seed: int, amplitude: float = 0.01, mean: float = 0.5) -> np.ndarray:
    """c = mean everywhere plus, inside (phi >= 0.5), uniform noise
    amplitude (2 rand(MersenneTwister(seed), n, n) - 1) with its interior mean
    removed (core_shell.jl:31-35)."""
    noise = amplitude * (2.0 * julia_rand(seed, phi.shape[1], phi.shape[0]) - 1.0)
    inside = phi >= 0.5
    c = np.full(phi.shape, mean, dtype=np.float64)
    if inside.any():
        noise = noise - noise[inside].mean()
        c[inside] += noise[inside]
    return c


def whole_field_noise(n: int, seed: int, mean: float = 0.5, amplitude: float = 0.01) -> np.ndarray:
    """c0 = mean + amplitude (2 rand(MersenneTwister(seed), n, n) - 1) on every point."""
    return mean + amplitude * (2.0 * julia_rand(seed, n) - 1.0)


def initial_fields(n: int, spacing: float = 1.0, radius: float = 70.0, width: float = 4.0, seed: int = 5749):
    """``initial_fields`` of core_shell.jl:27-37: returns (c, phi)."""
    phi = particle_disc(n, spacing, radius, width)
    return interior_noise(phi, seed), phi


# ---- the shape set and the counter-based noise of esc_particle_device / esc_noise_device ----

def _profile(r, R, w):
    return 0.5 * (1.0 - np.tanh((r - R) / w))


def particle(shape: str, n: int, params, width: float = 2.0, spacing: float = 1.0) -> np.ndarray:
    """Host mirror of esc_particle_device (shapes and parameters as in include/esc.h)."""
    p = list(params) + [0.0] * (4 - len(params))
    x = _centred(n, spacing).reshape(1, n)
    y = _centred(n, spacing).reshape(n, 1)
    r = np.sqrt(x * x + y * y)
    w = width
    if shape == "disc":
        return _profile(r, p[0], w) + 0.0 * x
    if shape == "band":
        return 0.5 * (np.tanh((y - p[0]) / w) - np.tanh((y - p[1]) / w)) + 0.0 * x
    if shape == "ellipse":
        return _profile(np.sqrt((x * p[1] / p[0]) ** 2 + y * y), p[1], w)
    if shape == "annulus":
        return _profile(r, p[1], w) - _profile(r, p[0], w)
    if shape == "squircle":
        return _profile(np.sqrt(np.sqrt(x ** 4 + y ** 4)), p[0], w)
    if shape == "elliptic_shell":
        return _profile(np.sqrt((x * p[1] / p[0]) ** 2 + y * y), p[1], w) - _profile(r, p[2], w)
    if shape == "elliptic_hole":
        return _profile(r, p[0], w) - _profile(np.sqrt((x * p[2] / p[1]) ** 2 + y * y), p[2], w)
    raise ValueError(f"unknown shape {shape!r}")


def splitmix_uniform(seed: int, count: int) -> np.ndarray:
    """u_k in [0, 1) for k < count: SplitMix64 of state seed + (k+1) * golden gamma, top 53 bits."""
    with np.errstate(over="ignore"):
        k = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + k * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def counter_noise(n: int, seed: int, phi=None, mean: float = 0.5, amplitude: float = 0.01) -> np.ndarray:
    """Host mirror of esc_noise_device."""
    e = (amplitude * (2.0 * splitmix_uniform(seed, n * n) - 1.0)).reshape(n, n)
    if phi is None:
        return mean + e
    inside = np.asarray(phi) >= 0.5
    shift = e[inside].mean() if inside.any() else 0.0
    return np.where(inside, mean + (e - shift), mean)
