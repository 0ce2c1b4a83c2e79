"""CPU oracle for the fixed-particle Cahn-Hilliard time loop (FP64, NumPy + scipy.fft).

TEST INFRASTRUCTURE ONLY.  This module is the checker: the tests, the smoke
check and the CPU-baseline leg of the benchmark may import it; the product path
(the CUDA library and its Python binding) never does.

It restates, function by function, the Julia model of the reference
(``core_shell.jl`` of saswataiith/embedded-spinodal-core-shell-julia) in NumPy.
Each function cites the line range it follows.  The FFT is pocketfft (via
``scipy.fft``) instead of FFTW 3.3.12 (FFTW_jll 3.3.12+0 behind FFTW.jl 1.10.0,
reference ``Manifest.toml:48-58``); both compute the unnormalised forward DFT
and the 1/N-normalised inverse, so results agree to rounding.

Memory layout.  Julia stores an n-by-n ``Matrix{Float64}`` column-major with
dimension 1 (index ``i``, the x direction, the one ``kx`` varies along)
contiguous.  Here every field is a C-ordered NumPy array ``a[j, i]`` of shape
``(n, n)``: axis 1 is x (contiguous), axis 0 is y.  The bytes are therefore
identical to the Julia matrix, which is what crosses the C ABI.

Noise.  ``initial_fields`` draws the reference's own stream,
``rand(MersenneTwister(seed), n, n)`` (core_shell.jl:32), from the restatement
of Julia's seeding and dSFMT-19937 in ``julia_rng.py``.

Pinning.  The reference ships no output fields, but ``check-results.txt:1-7``
records the numbers its ``checks.jl`` printed for exactly these inputs.  With
the reproduced noise this oracle matches them: the initial energies
329.48858453024934 (64^2, radius 16; exactly) and 4406.5104552251505 (256^2;
2e-16), the final energies of the three time-step runs and of the 256^2 run
(<= 2e-15 relative), the final composition ranges (<= 1.2e-13) and the two RMS
differences between time steps (<= 2.1e-11), see ``tests/test_oracle.py``.  It
also passes the reference's own identities (``checks.jl:11-29``) and agrees to
~1e-14 with a second, independent restatement in C with its own FFT
(``core_shell_oracle.c``).
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np
import scipy.fft as sfft

from . import julia_rng

_WORKERS = int(os.environ.get("ESC_ORACLE_WORKERS", "1"))


def set_workers(workers: int) -> None:
    """Thread count used by every FFT of the oracle (scipy.fft ``workers``)."""
    global _WORKERS
    _WORKERS = max(1, int(workers))


def _fft(a):
    return sfft.fft2(a, workers=_WORKERS)


def _ifft(a):
    return sfft.ifft2(a, workers=_WORKERS)


@dataclasses.dataclass(frozen=True)
class Parameters:
    """Model constants, defaults as ``core_shell.jl:4-15``."""

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

    def as_tuple(self):
        return (self.A, self.B, self.chi, self.P, self.ca, self.cb, self.cc,
                self.kappa, self.mobility, self.Q)


@dataclasses.dataclass
class Grid:
    kx: np.ndarray  # (1, n): derivative wavenumber along x (axis 1), Nyquist zeroed
    ky: np.ndarray  # (n, 1): derivative wavenumber along y (axis 0), Nyquist zeroed
    k2: np.ndarray  # (n, n): |k|^2 with the Nyquist kept
    spacing: float


@dataclasses.dataclass
class Shape:
    h: np.ndarray
    g: np.ndarray
    M: np.ndarray


class NonFiniteError(RuntimeError):
    """Raised like ``error("Non-finite composition at step $s")`` (core_shell.jl:93)."""

    def __init__(self, step: int):
        super().__init__(f"Non-finite composition at step {step}")
        self.step = step


def wavenumbers(n: int, spacing: float) -> np.ndarray:
    """``2pi .* fftfreq(n, 1/spacing)`` (core_shell.jl:18)."""
    return 2.0 * np.pi * np.fft.fftfreq(n, d=spacing)


def make_grid(n: int, spacing: float) -> Grid:
    """core_shell.jl:17-25.  The first-derivative wavenumber has its even-n
    Nyquist entry set to zero (:20); ``k2`` keeps the full k^2 (:23)."""
    k = wavenumbers(n, spacing)
    dk = k.copy()
    if n % 2 == 0:
        dk[n // 2] = 0.0
    kx = dk.reshape(1, n)
    ky = dk.reshape(n, 1)
    k2 = (k ** 2).reshape(1, n) + (k ** 2).reshape(n, 1)
    return Grid(kx=kx, ky=ky, k2=k2, spacing=float(spacing))


def particle_disc(n: int, spacing: float = 1.0, radius: float = 70.0,
                  width: float = 4.0) -> np.ndarray:
    """The tanh disc of core_shell.jl:29-30, centred on index n÷2 (0-based)."""
    idx = (np.arange(n) - n // 2) * spacing
    r = np.hypot(idx.reshape(1, n), idx.reshape(n, 1))
    return 0.5 * (1.0 - np.tanh((r - radius) / width))


def particle_ellipse(n: int, a: float, b: float, width: float,
                     spacing: float = 1.0) -> np.ndarray:
    """Elliptical particle phi = 0.5(1 - tanh((sqrt((x b/a)^2 + y^2) - b)/w)),
    x along axis 1 with semi-axis a, y along axis 0 with semi-axis b, centred
    on index n÷2 like the disc."""
    idx = (np.arange(n) - n // 2) * spacing
    x = idx.reshape(1, n)
    y = idx.reshape(n, 1)
    r = np.sqrt((x * b / a) ** 2 + y ** 2)
    return 0.5 * (1.0 - np.tanh((r - b) / width))


def interior_noise(phi: np.ndarray, seed: int, amplitude: float = 0.01,
                   mean: float = 0.5) -> np.ndarray:
    """core_shell.jl:31-35: c = mean inside and out; inside (phi >= 0.5) add
    amplitude (2 rand(MersenneTwister(seed), n, n) - 1) whose interior mean is
    removed."""
    noise = amplitude * (2.0 * julia_rng.rand_matrix(seed, phi.shape[1], phi.shape[0]) - 1.0)
    inside = phi >= 0.5
    c = np.full(phi.shape, mean, dtype=np.float64)
    if inside.any():
        noise = noise - noise[inside].mean()
        c[inside] += noise[inside]
    return c


def whole_field_noise(n: int, seed: int, mean: float = 0.5,
                      amplitude: float = 0.01) -> np.ndarray:
    """c0 = mean + amplitude (2 rand(MersenneTwister(seed), n, n) - 1) over the whole field."""
    return mean + amplitude * (2.0 * julia_rng.rand_matrix(seed, n) - 1.0)


def initial_fields(n: int, spacing: float = 1.0, radius: float = 70.0,
                   width: float = 4.0, seed: int = 5749):
    """core_shell.jl:27-37: returns (c, phi) with the reference's noise stream."""
    phi = particle_disc(n, spacing, radius, width)
    return interior_noise(phi, seed), phi


def geometry(phi: np.ndarray, p: Parameters) -> Shape:
    """core_shell.jl:39-43."""
    h = phi ** 3 * (10.0 - 15.0 * phi + 6.0 * phi ** 2)
    g = phi ** 2 * (1.0 - phi) ** 2
    return Shape(h=h, g=g, M=p.mobility * h)


def bulk_energy(c, shape: Shape, p: Parameters):
    """core_shell.jl:45-49."""
    h, g = shape.h, shape.g
    return (p.A * (1 - h) * (c - p.ca) ** 2
            + p.B * h * (c - p.cb) ** 2 * (c - p.cc) ** 2
            + p.P * (1 - p.chi * c) * g)


def bulk_derivative(c, shape: Shape, p: Parameters):
    """core_shell.jl:51-55."""
    h, g = shape.h, shape.g
    return (2 * p.A * (1 - h) * (c - p.ca)
            + 2 * p.B * h * (c - p.cb) * (c - p.cc) * (2 * c - p.cb - p.cc)
            - p.chi * p.P * g)


def chemical_potential(c, shape: Shape, grid: Grid, p: Parameters):
    """core_shell.jl:57-60: f'(c) + Re IFFT(2 kappa k^2 FFT(c))."""
    return bulk_derivative(c, shape, p) + np.real(
        _ifft(2 * p.kappa * grid.k2 * _fft(c)))


def transport_rate(c, shape: Shape, grid: Grid, p: Parameters):
    """core_shell.jl:62-70.  Returns (FFT of div(M grad mu), dissipation)."""
    mu_hat = _fft(chemical_potential(c, shape, grid, p))
    grad_x = np.real(_ifft(1j * grid.kx * mu_hat))
    grad_y = np.real(_ifft(1j * grid.ky * mu_hat))
    divergence_hat = (1j * grid.kx * _fft(shape.M * grad_x)
                      + 1j * grid.ky * _fft(shape.M * grad_y))
    dissipation = np.sum(shape.M * (grad_x ** 2 + grad_y ** 2)) * grid.spacing ** 2
    return divergence_hat, dissipation


def step(c, shape: Shape, grid: Grid, p: Parameters, dt: float):
    """core_shell.jl:72-76: the stabilised semi-implicit Fourier update."""
    rate, _ = transport_rate(c, shape, grid, p)
    denominator = 1 + 2 * p.Q * p.kappa * grid.k2 ** 2 * dt
    return np.real(_ifft(_fft(c) + dt * rate / denominator))


def energy(c, shape: Shape, grid: Grid, p: Parameters) -> float:
    """core_shell.jl:78-82 (Parseval; the Nyquist mode is included)."""
    gradient_energy = p.kappa * np.sum(grid.k2 * np.abs(_fft(c)) ** 2) / c.size
    return float((np.sum(bulk_energy(c, shape, p)) + gradient_energy)
                 * grid.spacing ** 2)


def run_simulation(c0, phi, dt: float = 0.01, steps: int = 1000,
                   spacing: float = 1.0, p: Parameters = Parameters()):
    """core_shell.jl:84-103 without the CSV output.

    Returns ``(c, history)``; ``history`` is ``(steps+1, 6)`` with rows
    ``[s*dt, mean c, energy, min c, max c, dissipation]`` recorded before the
    step, the step taken only while ``s < steps``.  A non-finite field raises
    :class:`NonFiniteError` after its row is recorded, as at :93.
    """
    c0 = np.asarray(c0, dtype=np.float64)
    n = c0.shape[0]
    grid = make_grid(n, spacing)
    shape = geometry(np.asarray(phi, dtype=np.float64), p)
    c = c0.copy()
    history = np.zeros((steps + 1, 6))
    for s in range(steps + 1):
        _, dissipation = transport_rate(c, shape, grid, p)
        history[s, :] = [s * dt, c.mean(), energy(c, shape, grid, p),
                         c.min(), c.max(), dissipation]
        if not np.all(np.isfinite(c)):
            raise NonFiniteError(s)
        if s < steps:
            c = step(c, shape, grid, p, dt)
    return c, history
