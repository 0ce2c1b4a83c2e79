"""Output and restart formats around the stepper (host side).

`write_results` writes the three files of the reference's `run_simulation`
(core_shell.jl:96-101): ``history.csv`` (steps+1 rows of
``[t, mean c, energy, min c, max c, dissipation]``), ``composition.csv`` and
``particle.csv``, comma-separated like Julia's ``writedlm(path, A, ',')``.  The
fields are written in Julia's row order: CSV row i holds the matrix row
``A[i, :]``, i.e. fixed x (the first, contiguous index) and increasing y, which
for a C-ordered array ``a[y, x]`` is column i.  Numbers use the shortest
representation that reads back to the same double, in the style Julia prints
Float64 (``0.5``, ``1.0e-5``, ``1.0e6``); Julia is not available to byte-compare
the text, so the guarantee is numerical: every value reads back exactly.

The coupled 3-D model writes configuration files in the layout of the reference's
3-D program (original/2023-3d/out_conf.cu:39-43): ``conf.%09d`` named by the step,
holding c and then phi as raw float64 in the order a[k + nz*(j + ny*i)] (z
contiguous), with no header; the grid shape travels separately
(`write_conf3d` / `read_conf3d`).

The restart format is a raw little-endian binary file: a 64-byte header
(magic ``ESCRST01``, int32 n, int32 flags, int64 step, float64 dt, float64 dx,
float64 time, 16 reserved bytes) followed by c (n*n float64, the bytes of the
Julia matrix) and, when flag bit 0 is set, phi in the same layout.
"""
from __future__ import annotations

import os
import struct
from typing import Optional, Tuple

import numpy as np

_MAGIC = b"ESCRST01"
_HEADER = struct.Struct("<8siiqddd16s")
assert _HEADER.size == 64


def julia_float(x: float) -> str:
    """Shortest round-trip text of a Float64 in the style of Julia's `print`:
    plain decimal for 1e-4 <= |x| < 1e6 (and 0), otherwise mantissa 'e' exponent,
    integral values keeping '.0'."""
    x = float(x)
    if x != x:
        return "NaN"
    if x in (float("inf"), float("-inf")):
        return "Inf" if x > 0 else "-Inf"
    if x == 0.0:
        return "-0.0" if np.signbit(x) else "0.0"
    r = repr(x)  # shortest round-trip digits
    mant, _, exp = r.partition("e")
    digits_exp = int(exp) if exp else 0
    # normalise to digits and a decimal exponent
    sign = "-" if mant.startswith("-") else ""
    mant = mant.lstrip("-")
    if "." in mant:
        ip, fp = mant.split(".")
    else:
        ip, fp = mant, ""
    digits = (ip + fp).lstrip("0")
    lead_zeros = len(ip + fp) - len((ip + fp).lstrip("0"))
    point = len(ip) - lead_zeros + digits_exp  # position of the decimal point within `digits`
    digits = digits.rstrip("0") or "0"
    a = abs(x)
    if 1e-4 <= a < 1e6:
        if point <= 0:
            return sign + "0." + "0" * (-point) + digits
        if point >= len(digits):
            return sign + digits + "0" * (point - len(digits)) + ".0"
        return sign + digits[:point] + "." + digits[point:]
    e = point - 1
    m = digits[0] + "." + (digits[1:] or "0")
    return f"{sign}{m}e{e}"


def _write_matrix(path: str, rows) -> None:
    with open(path, "w") as f:
        for row in rows:
            f.write(",".join(julia_float(v) for v in row))
            f.write("\n")


def write_history_csv(path: str, history: np.ndarray) -> None:
    """history: (steps+1, 6) as returned by run_simulation."""
    h = np.asarray(history, dtype=np.float64)
    if h.ndim != 2 or h.shape[1] != 6:
        raise ValueError(f"history must have shape (steps+1, 6), got {h.shape}")
    _write_matrix(path, h)


def write_field_csv(path: str, a: np.ndarray) -> None:
    """A field a[y, x] written as the Julia matrix A[x, y] by writedlm (row = fixed x)."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError("field must be 2-D")
    _write_matrix(path, a.T)


def read_field_csv(path: str) -> np.ndarray:
    """Inverse of write_field_csv (also reads a Julia-written composition.csv)."""
    return np.loadtxt(path, delimiter=",", ndmin=2).T.copy()


def write_results(directory: str, c: np.ndarray, history: np.ndarray, phi: np.ndarray) -> None:
    """The three files of core_shell.jl:96-101 in `directory` (created if needed)."""
    os.makedirs(directory, exist_ok=True)
    write_history_csv(os.path.join(directory, "history.csv"), history)
    write_field_csv(os.path.join(directory, "composition.csv"), c)
    write_field_csv(os.path.join(directory, "particle.csv"), phi)


def save_restart(path: str, c: np.ndarray, step: int, dt: float, dx: float = 1.0,
                 phi: Optional[np.ndarray] = None) -> None:
    c = np.ascontiguousarray(c, dtype="<f8")
    if c.ndim != 2 or c.shape[0] != c.shape[1]:
        raise ValueError("c must be square")
    n = c.shape[0]
    flags = 0
    if phi is not None:
        phi = np.ascontiguousarray(phi, dtype="<f8")
        if phi.shape != c.shape:
            raise ValueError("phi must match c")
        flags |= 1
    with open(path, "wb") as f:
        f.write(_HEADER.pack(_MAGIC, n, flags, int(step), float(dt), float(dx), float(step) * float(dt), b"\0" * 16))
        f.write(c.tobytes())
        if phi is not None:
            f.write(phi.tobytes())


def load_restart(path: str) -> Tuple[np.ndarray, Optional[np.ndarray], dict]:
    """Returns (c, phi or None, {"step", "dt", "dx", "time"})."""
    with open(path, "rb") as f:
        head = f.read(_HEADER.size)
        if len(head) != _HEADER.size:
            raise ValueError("truncated restart header")
        magic, n, flags, step, dt, dx, t, _ = _HEADER.unpack(head)
        if magic != _MAGIC:
            raise ValueError("not a restart file")
        if n <= 0:
            raise ValueError("bad grid size in restart header")
        body = f.read()
    need = n * n * 8 * (2 if flags & 1 else 1)
    if len(body) != need:
        raise ValueError(f"restart body has {len(body)} bytes, expected {need}")
    c = np.frombuffer(body[: n * n * 8], dtype="<f8").reshape(n, n).copy()
    phi = np.frombuffer(body[n * n * 8:], dtype="<f8").reshape(n, n).copy() if flags & 1 else None
    return c, phi, {"step": int(step), "dt": float(dt), "dx": float(dx), "time": float(t)}


def conf3d_name(step: int) -> str:
    """File name of a 3-D configuration after `step` steps: ``conf.%09d`` (out_conf.cu:39)."""
    return "conf.%09d" % int(step)


def write_conf3d(directory: str, step: int, c: np.ndarray, phi: np.ndarray) -> str:
    """Writes c then phi (float64, C order of shape (nx, ny, nz), i.e. z contiguous) to
    ``directory/conf.%09d`` like the reference's Output_conf (out_conf.cu:39-43); returns the path."""
    c = np.ascontiguousarray(c, dtype="<f8")
    phi = np.ascontiguousarray(phi, dtype="<f8")
    if c.shape != phi.shape or c.ndim != 3:
        raise ValueError("c and phi must be 3-D arrays of one shape")
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, conf3d_name(step))
    with open(path, "wb") as f:
        f.write(c.tobytes())
        f.write(phi.tobytes())
    return path


def read_conf3d(path: str, shape: Tuple[int, int, int]) -> Tuple[np.ndarray, np.ndarray]:
    """Reads a configuration file of `write_conf3d` (or of the reference's 3-D program)
    for a grid of `shape` = (nx, ny, nz); returns (c, phi)."""
    n = int(np.prod(shape))
    raw = np.fromfile(path, dtype="<f8")
    if raw.size != 2 * n:
        raise ValueError(f"{path}: {raw.size} values, expected {2 * n} for shape {tuple(shape)}")
    return raw[:n].reshape(shape).copy(), raw[n:].reshape(shape).copy()
