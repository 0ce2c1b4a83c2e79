"""Generates the golden fixtures in this directory from the CPU oracle.

Run from the repository root:  python tests/golden/make_golden.py
Each fixture holds the inputs (c0, phi, parameters, dt, steps; c0 from the
reference's own noise stream, initial_fields) and the oracle's
outputs (final c, history) of a short run of run_simulation
(core_shell.jl:84-103).  The GPU parity tests compare the CUDA library with
these files; the CPU tests re-run the oracle and compare it with them, which
pins the oracle against accidental drift.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import core_shell_oracle as orc  # noqa: E402
from oracle import coupled_oracle as cpl  # noqa: E402

CASES = [
    # name, n, radius, width, seed, steps, dt, params overrides
    ("disc16_r4", 16, 4.0, 1.0, 1, 12, 0.01, {}),
    ("disc48_r12", 48, 12.0, 2.0, 2, 40, 0.01, {"P": 6.0, "chi": 0.6}),
    ("disc64_r16", 64, 16.0, 4.0, 5749, 100, 0.01, {}),
    ("disc96_r24_dt005", 96, 24.0, 2.0, 3, 60, 0.005, {"kappa": 3.0, "Q": 0.7}),
]


def make(name, n, radius, width, seed, steps, dt, over):
    c0, phi = orc.initial_fields(n, radius=radius, width=width, seed=seed)
    p = orc.Parameters(**over)
    c, hist = orc.run_simulation(c0, phi, dt=dt, steps=steps, p=p)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), c0=c0, phi=phi, c=c, history=hist,
                        params=np.array(p.as_tuple()), dt=dt, steps=steps)


def make_coupled():
    """The coupled c-phi model (original/2023-3d restated): a 24 x 16 x 32 grid with
    unequal spacings and non-default constants, 25 steps."""
    p = cpl.CoupledParameters(P=5.0, kappa_phi=6.0, relax=0.01, A0=0.1)
    c0, phi0 = cpl.initial_fields(24, 16, 32, 6.0, seed=7, p=p)
    spacing = (1.0, 0.9, 1.1)
    c, phi, hist, done, reason = cpl.run(c0, phi0, p, 0.01, 25, spacing=spacing)
    names = list(vars(p).keys())
    np.savez_compressed(os.path.join(HERE, "coupled_24x16x32.npz"), c0=c0, phi0=phi0, c=c, phi=phi, history=hist,
                        param_names=np.array(names), param_values=np.array([vars(p)[k] for k in names]),
                        dt=0.01, steps=25, spacing=np.array(spacing))


if __name__ == "__main__":
    for case in CASES:
        make(*case)
        print("wrote", case[0])
    make_coupled()
    print("wrote coupled_24x16x32")
