"""CPU oracle for gradients of the fixed-particle Cahn-Hilliard time loop (FP64).

TEST INFRASTRUCTURE ONLY (the checker of the CUDA adjoint; never on the product path).

The loss is that of the calibration configuration:
    L = 1/2 * sum_x (c_T - c_target)^2 + lam_F * F[c_T]
with c_T after `steps` applications of the reference step (core_shell.jl:72-76)
and F the reference energy (core_shell.jl:78-82).  Gradients are taken with
respect to c0 and theta = (P, chi, kappa, M0).

Three independent evaluations are provided:
  * `gradient`  -- reverse mode (the transposed step, restated below);
  * `jvp`       -- forward mode: the tangent-linear step, i.e. dual numbers
                   propagated through every operation of the reference step;
  * `loss`      -- for central finite differences.

Writing S = IFFT diag(1/den) FFT, D_x = IFFT diag(i k_x) FFT (derivative
Nyquist zeroed, core_shell.jl:20), L = -IFFT diag(k2) FFT and M = M0 h(phi),
the step is  c' = c + dt S div(M grad mu(c)),  mu = f'(c) - 2 kappa L c.
All four operators are real; S, L and div(M grad .) are symmetric and D_x is
antisymmetric, so the transposed step is
    a = dt S lam,  g = div(M grad a),  lam_prev = lam + f''(c) g - 2 kappa L g,
and the parameter sensitivities of one step are
    dP = sum g (-chi gphi),  dchi = sum g (-P gphi),
    dkappa = sum g IFFT(2 k2 c^) + sum lam IFFT((c'^ - c^)(-2 Q k2^2 dt)/den),
    dM0 = sum lam (c' - c) / M0      (the update is linear in M0).
"""
from __future__ import annotations

import numpy as np

from . import core_shell_oracle as orc

THETA = ("P", "chi", "kappa", "mobility")


def _fft(a):
    return orc._fft(a)


def _ifft(a):
    return orc._ifft(a)


def _with(p: orc.Parameters, **kw) -> orc.Parameters:
    d = {f: getattr(p, f) for f in ("A", "B", "chi", "P", "ca", "cb", "cc", "kappa", "mobility", "Q")}
    d.update(kw)
    return orc.Parameters(**d)


def bulk_second_derivative(c, shape: orc.Shape, p: orc.Parameters):
    """d^2 f / dc^2 of core_shell.jl:45-49."""
    h = shape.h
    e = 2 * c - p.cb - p.cc
    return (2 * p.A * (1 - h)
            + 2 * p.B * h * ((c - p.cc) * e + (c - p.cb) * e + 2 * (c - p.cb) * (c - p.cc)))


def _den(grid: orc.Grid, p: orc.Parameters, dt: float):
    return 1 + 2 * p.Q * p.kappa * grid.k2 ** 2 * dt


def forward_states(c0, phi, steps, dt, p, spacing=1.0):
    """All states c_0 .. c_steps of the reference step."""
    n = c0.shape[0]
    grid = orc.make_grid(n, spacing)
    shape = orc.geometry(phi, p)
    cs = [np.array(c0, dtype=np.float64)]
    for _ in range(steps):
        cs.append(orc.step(cs[-1], shape, grid, p, dt))
    return cs


def loss(c0, phi, steps, dt, c_target, lam_F, p, spacing=1.0):
    cs = forward_states(c0, phi, steps, dt, p, spacing)
    grid = orc.make_grid(c0.shape[0], spacing)
    shape = orc.geometry(phi, p)
    cT = cs[-1]
    return 0.5 * float(np.sum((cT - c_target) ** 2)) + lam_F * orc.energy(cT, shape, grid, p)


def energy_theta_gradient(c, phi, p, spacing=1.0):
    """dF/d(P, chi, kappa, M0) at fixed c (core_shell.jl:78-82)."""
    grid = orc.make_grid(c.shape[0], spacing)
    shape = orc.geometry(phi, p)
    dx2 = spacing ** 2
    g = shape.g
    dP = float(np.sum((1 - p.chi * c) * g)) * dx2
    dchi = float(np.sum(-p.P * c * g)) * dx2
    dkappa = float(np.sum(grid.k2 * np.abs(_fft(c)) ** 2) / c.size) * dx2
    return np.array([dP, dchi, dkappa, 0.0])


def adjoint_step(lam, c, c_next, shape, grid, p, dt):
    """lam_prev and the theta sensitivities of one step (see module docstring)."""
    den = _den(grid, p, dt)
    lam_hat = _fft(lam)
    a_hat = dt * lam_hat / den
    ax = np.real(_ifft(1j * grid.kx * a_hat))
    ay = np.real(_ifft(1j * grid.ky * a_hat))
    g_hat = 1j * grid.kx * _fft(shape.M * ax) + 1j * grid.ky * _fft(shape.M * ay)
    g = np.real(_ifft(g_hat))
    lam_prev = lam + bulk_second_derivative(c, shape, p) * g + np.real(_ifft(2 * p.kappa * grid.k2 * g_hat))
    c_hat = _fft(c)
    d_hat = _fft(c_next) - c_hat
    dP = float(np.sum(g * (-p.chi * shape.g)))
    dchi = float(np.sum(g * (-p.P * shape.g)))
    dkappa = float(np.sum(g * np.real(_ifft(2 * grid.k2 * c_hat)))
                   + np.sum(lam * np.real(_ifft(d_hat * (-2 * p.Q * grid.k2 ** 2 * dt) / den))))
    dM0 = float(np.sum(lam * (c_next - c)) / p.mobility)
    return lam_prev, np.array([dP, dchi, dkappa, dM0])


def gradient(c0, phi, steps, dt, c_target, lam_F, p, spacing=1.0):
    """(L, dL/dc0, dL/dtheta) by reverse mode over stored states."""
    n = c0.shape[0]
    grid = orc.make_grid(n, spacing)
    shape = orc.geometry(phi, p)
    cs = forward_states(c0, phi, steps, dt, p, spacing)
    cT = cs[-1]
    L = 0.5 * float(np.sum((cT - c_target) ** 2)) + lam_F * orc.energy(cT, shape, grid, p)
    lam = (cT - c_target) + lam_F * orc.chemical_potential(cT, shape, grid, p) * spacing ** 2
    dtheta = lam_F * energy_theta_gradient(cT, phi, p, spacing)
    for s in range(steps - 1, -1, -1):
        lam, d = adjoint_step(lam, cs[s], cs[s + 1], shape, grid, p, dt)
        dtheta = dtheta + d
    return L, lam, dtheta


def tangent_step(c, cdot, shape, grid, p, dt, theta_dot):
    """Tangent-linear (dual-number) image of one reference step."""
    Pd, chid, kappad, M0d = theta_dot
    den = _den(grid, p, dt)
    c_hat = _fft(c)
    cd_hat = _fft(cdot)
    fpp = bulk_second_derivative(c, shape, p)
    mu = orc.chemical_potential(c, shape, grid, p)
    mu_dot = (fpp * cdot + np.real(_ifft(2 * p.kappa * grid.k2 * cd_hat))
              + np.real(_ifft(2 * kappad * grid.k2 * c_hat))
              - p.chi * shape.g * Pd - p.P * shape.g * chid)
    mu_hat, mud_hat = _fft(mu), _fft(mu_dot)
    gx, gy = np.real(_ifft(1j * grid.kx * mu_hat)), np.real(_ifft(1j * grid.ky * mu_hat))
    gxd, gyd = np.real(_ifft(1j * grid.kx * mud_hat)), np.real(_ifft(1j * grid.ky * mud_hat))
    Md = M0d * shape.h
    div = 1j * grid.kx * _fft(shape.M * gx) + 1j * grid.ky * _fft(shape.M * gy)
    div_dot = (1j * grid.kx * _fft(shape.M * gxd + Md * gx) + 1j * grid.ky * _fft(shape.M * gyd + Md * gy))
    den_dot = 2 * p.Q * kappad * grid.k2 ** 2 * dt
    c_new = np.real(_ifft(c_hat + dt * div / den))
    cd_new = np.real(_ifft(cd_hat + dt * div_dot / den - dt * div * den_dot / den ** 2))
    return c_new, cd_new


def jvp(c0, phi, steps, dt, c_target, lam_F, p, c0_dot, theta_dot, spacing=1.0):
    """Directional derivative dL[c0_dot, theta_dot] by forward (dual-number) mode."""
    n = c0.shape[0]
    grid = orc.make_grid(n, spacing)
    shape = orc.geometry(phi, p)
    c, cd = np.array(c0, dtype=np.float64), np.array(c0_dot, dtype=np.float64)
    for _ in range(steps):
        c, cd = tangent_step(c, cd, shape, grid, p, dt, theta_dot)
    mu = orc.chemical_potential(c, shape, grid, p)
    ld = float(np.sum((c - c_target) * cd)) + lam_F * float(np.sum(mu * cd)) * spacing ** 2
    ld += lam_F * float(np.dot(energy_theta_gradient(c, phi, p, spacing), theta_dot))
    return ld


def perturbed(p: orc.Parameters, k: int, h: float) -> orc.Parameters:
    return _with(p, **{THETA[k]: getattr(p, THETA[k]) + h})
