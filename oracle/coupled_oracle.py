"""CPU oracle for the coupled c-phi model (conserved c, Allen-Cahn phi) in 3-D.

TEST INFRASTRUCTURE ONLY: the tests and the benchmark's CPU-baseline leg import
this module as the checker; the library never does.

A NumPy restatement, operation for operation, of the step of the reference's
2023 3-D program (original/2023-3d/evolve.cu:55-186 with the kernels of
original/2023-3d/EvoKernels.h).  Only the mathematics is restated; arrays use
the reference's memory order a[i, j, k] = a[k + nz*(j + ny*i)] (x slowest, z
contiguous), i.e. C-ordered NumPy arrays of shape (nx, ny, nz).

Per step (the reference's order):
  1. local terms from the real fields (EvoKernels.h:1-37, kernel_cphi_der):
       h = phi^3 (10 - 15 phi + 6 phi^2),   g = phi^2 (1 - phi)^2,
       h' = 30 (phi^2 - 2 phi^3 + phi^4),   g' = 2 phi - 6 phi^2 + 4 phi^3,
       df/dc   = 2A(1-h)(c-ca) + 2Bh(c-cb1)(c-cb2)(2c-cb1-cb2) - chi P g,
       df/dphi = -h'(A(c-ca)^2 + A0) + h' B (c-cb1)^2 (c-cb2)^2 + (1 - chi c) P g',
       M       = mobility h;
  2. mu^ = FFT(df/dc) + 2 kappa_c k^2 c^       (EvoKernels.h:38-58, Compute_mu;
     k^2 keeps the Nyquist wavenumber, main.cu:139-175 kx2/ky2/kz2);
  3. mu = Re IFFT(mu^) / N                      (evolve.cu:102-106, Muscaling);
  4. div = sum_a D_a(M D_a mu), D_a the fourth-order central difference
     (-f[+2] + 8 f[+1] - 8 f[-1] + f[-2]) / (12 h_a), periodic
     (EvoKernels.h:74-419, ComputeGradmu_* and ComputeGrad_*);
  5. c^' = (dt div^ + lhs c^) / lhs,  lhs = 1 + 2 Q kappa_c k^4 dt,
     phi^' = (phi^ - L dt FFT(df/dphi)) / (1 + 2 L kappa_phi k^2 dt)
     (EvoKernels.h:432-470, kernel_comp_phi);
  6. mass check |c^'(0)/N - mean c0| > COMPERR stops the run
     (evolve.cu:145-155, COMPERR = 1e-8 in binary.h:14);
  7. c = Re IFFT(c^')/N, phi = Re IFFT(phi^')/N (evolve.cu:157-160, Normalization);
     composition bounds -0.4 <= c <= 1.4 (EvoKernels.h:489-508, Bounds) and
     convergence max|c - c_prev| <= Tolerance (evolve.cu:168-181) end the loop.

The reference passes dy to the z-gradient of mu (evolve.cu:124, "ComputeGradmu_z
... dy"), an error its numerical review names; `z_grad_spacing="dz"` (the
default) uses dz, `"dy"` reproduces the reference's call.  They agree when
dy == dz.
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft

# stop reasons of `run` (and of the library's coupled run)
RUNNING, CONVERGED, OUT_OF_BOUNDS, MASS_ERROR, NONFINITE = 0, 1, 2, 3, 4
C_LOW, C_HIGH = -0.4, 1.4            # EvoKernels.h:499
COMPERR = 1.0e-8                      # binary.h:14


class CoupledParameters:
    """Model constants of the coupled program (original/2023-3d/InputParams:13-22)."""

    def __init__(self, A=2.0, B=1.0, chi=0.5, P=6.0, ca=0.5, cb1=0.0, cb2=1.0, A0=0.08,
                 kappa_c=2.0, kappa_phi=10.0, mobility=1.0, relax=0.001, Q=0.5):
        self.A, self.B, self.chi, self.P = A, B, chi, P
        self.ca, self.cb1, self.cb2, self.A0 = ca, cb1, cb2, A0
        self.kappa_c, self.kappa_phi = kappa_c, kappa_phi
        self.mobility, self.relax, self.Q = mobility, relax, Q


def wavenumbers(n: int, h: float) -> np.ndarray:
    """kx2 of main.cu:139-160: i dk for i <= n/2 (the Nyquist kept, positive), (i - n) dk above."""
    dk = 2.0 * np.pi / (n * h)
    i = np.arange(n)
    return np.where(i <= n // 2, i, i - n).astype(np.float64) * dk


def k_squared(shape, spacing) -> np.ndarray:
    nx, ny, nz = shape
    dx, dy, dz = spacing
    kx, ky, kz = wavenumbers(nx, dx), wavenumbers(ny, dy), wavenumbers(nz, dz)
    return kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2


def fd4(f: np.ndarray, axis: int, h: float) -> np.ndarray:
    """Fourth-order central difference with periodic neighbours (EvoKernels.h:125, :296)."""
    p1, p2 = np.roll(f, -1, axis), np.roll(f, -2, axis)
    m1, m2 = np.roll(f, 1, axis), np.roll(f, 2, axis)
    return (-1.0 * p2 + 8.0 * p1 - 8.0 * m1 + m2) / (12.0 * h)


def local_terms(c: np.ndarray, phi: np.ndarray, p: CoupledParameters):
    """(df/dc, df/dphi, M) of kernel_cphi_der, EvoKernels.h:1-37."""
    h = phi * phi * phi * (10.0 - 15.0 * phi + 6.0 * phi * phi)
    g = (phi * phi) * (1.0 - phi) * (1.0 - phi)
    hp = 30.0 * (phi * phi - 2.0 * phi * phi * phi + phi * phi * phi * phi)
    gp = 2.0 * phi - 6.0 * phi * phi + 4.0 * phi * phi * phi
    dfdc = (2.0 * p.A * (1.0 - h) * (c - p.ca)
            + 2.0 * p.B * h * (c - p.cb1) * (c - p.cb2) * (2.0 * c - p.cb1 - p.cb2) - p.chi * p.P * g)
    dfdphi = (-1.0 * hp * (p.A * (c - p.ca) * (c - p.ca) + p.A0)
              + hp * p.B * (c - p.cb1) * (c - p.cb1) * (c - p.cb2) * (c - p.cb2)
              + (1.0 - p.chi * c) * p.P * gp)
    return dfdc, dfdphi, h * p.mobility


def divergence(mu: np.ndarray, M: np.ndarray, spacing, z_grad_spacing="dz") -> np.ndarray:
    """div(M grad mu) with fourth-order differences (EvoKernels.h:74-419, evolve.cu:108-130)."""
    dx, dy, dz = spacing
    dzg = dz if z_grad_spacing == "dz" else dy
    return (fd4(M * fd4(mu, 0, dx), 0, dx) + fd4(M * fd4(mu, 1, dy), 1, dy)
            + fd4(M * fd4(mu, 2, dzg), 2, dz))


def step(chat, phihat, c, phi, p: CoupledParameters, dt: float, spacing, k2=None, z_grad_spacing="dz"):
    """One step of evolve.cu:86-160; returns (c^', phi^', c', phi')."""
    if k2 is None:
        k2 = k_squared(c.shape, spacing)
    dfdc, dfdphi, M = local_terms(c, phi, p)
    muhat = sfft.fftn(dfdc) + 2.0 * p.kappa_c * k2 * chat
    mu = sfft.ifftn(muhat).real                    # ifftn includes the 1/N of Muscaling
    div = divergence(mu, M, spacing, z_grad_spacing)
    divhat = sfft.fftn(div)
    lhs = 1.0 + 2.0 * p.Q * p.kappa_c * k2 * k2 * dt
    chat_n = (dt * divhat + lhs * chat) / lhs
    lhse = 1.0 + 2.0 * p.relax * p.kappa_phi * k2 * dt
    phihat_n = (phihat - p.relax * dt * sfft.fftn(dfdphi)) / lhse
    return chat_n, phihat_n, sfft.ifftn(chat_n).real, sfft.ifftn(phihat_n).real


def history_row(t, c, phi, c_prev):
    """[t, mean c, mean phi, min c, max c, max |c - c_prev|] (the library's coupled history)."""
    return [t, float(np.mean(c)), float(np.mean(phi)), float(np.min(c)), float(np.max(c)),
            0.0 if c_prev is None else float(np.max(np.abs(c - c_prev)))]


def run(c0, phi0, p: CoupledParameters, dt: float, steps: int, spacing=(1.0, 1.0, 1.0),
        tolerance: float = 0.0, comperr: float = COMPERR, z_grad_spacing="dz"):
    """Up to `steps` steps from (c0, phi0).  Returns (c, phi, history, steps_done, reason).

    history has one row per recorded state (row s = after s steps, row 0 the input);
    the run ends early, like the reference's loop, when the mean composition drifts
    by more than comperr (the fields of the failing step are not kept, evolve.cu:149-154),
    when c leaves [-0.4, 1.4], or when max|c - c_prev| <= tolerance."""
    c = np.array(c0, dtype=np.float64)
    phi = np.array(phi0, dtype=np.float64)
    k2 = k_squared(c.shape, spacing)
    chat, phihat = sfft.fftn(c), sfft.fftn(phi)
    mean0 = float(np.sum(c)) / c.size               # alloycomp, evolve.cu:36-46
    hist = [history_row(0.0, c, phi, None)]
    reason, done = RUNNING, 0
    for s in range(steps):
        chat_n, phihat_n, c_n, phi_n = step(chat, phihat, c, phi, p, dt, spacing, k2, z_grad_spacing)
        if not abs(chat_n.flat[0].real / c.size - mean0) <= comperr:
            reason = MASS_ERROR
            break
        c_prev = c
        chat, phihat, c, phi = chat_n, phihat_n, c_n, phi_n
        done = s + 1
        hist.append(history_row(done * dt, c, phi, c_prev))
        if not np.all(np.isfinite(c)):
            reason = NONFINITE
            break
        if np.any(c < C_LOW) or np.any(c > C_HIGH):
            reason = OUT_OF_BOUNDS
            break
        if hist[-1][5] <= tolerance:
            reason = CONVERGED
            break
    return c, phi, np.array(hist), done, reason


def initial_fields(nx, ny, nz, radius, c_mean=0.5, noise=0.05, seed=2938, p: CoupledParameters | None = None,
                   phicutoff=0.5):
    """Sharp spherical particle and noisy composition of init_conf.cu:55-125 (flag 1):
    phi = 1 for r < R about (nx/2, ny/2, nz/2), else 0; inside (phi > phicutoff)
    c = c_mean (cb1 + cb2) + r - <r>, r uniform in [-noise, noise) with its mean over
    the particle removed; outside c = ca.  The uniform numbers come from NumPy's
    PCG64 (the reference draws them with cuRAND)."""
    p = p or CoupledParameters()
    i = np.arange(nx)[:, None, None] - nx // 2
    j = np.arange(ny)[None, :, None] - ny // 2
    k = np.arange(nz)[None, None, :] - nz // 2
    r = np.sqrt((i * i + j * j + k * k).astype(np.float64))
    phi = np.where(r < radius, 1.0, 0.0)
    rnd = (2.0 * np.random.default_rng(seed).random((nx, ny, nz)) - 1.0) * noise
    inside = phi > phicutoff
    mean = rnd[inside].mean() if inside.any() else 0.0
    c = np.where(inside, c_mean * (p.cb1 + p.cb2) + rnd - mean, p.ca)
    return c, phi
