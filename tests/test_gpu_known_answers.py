"""The FP64 drop-in against the numbers the reference itself printed.

check-results.txt:2-7 records what the reference's checks.jl printed for the
inputs of initial_fields(64; radius=16) and initial_fields(256) (core_shell.jl:27-37,
noise from rand(MersenneTwister(5749), n, n), reproduced here exactly): initial
and final energies, final composition ranges and the RMS differences between
time steps.  The CUDA library, run through the C ABI on those inputs, must give
them to 1e-10 relative (1e-9 for the RMS of a difference of two fields), and
must reproduce the committed golden fixtures (written by the oracle) to 1e-12.
"""
import os

import numpy as np
import pytest

import esc
from esc import fields

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

KNOWN_64 = {   # dt -> (E(t=0), E(t=10), min c, max c); check-results.txt:2-4
    0.01: (329.48858453024934, 290.1672693863404, 0.03738467482348276, 0.9430096320792813),
    0.005: (329.48858453024934, 290.15644231050993, 0.037201502506359285, 0.9430283569784008),
    0.0025: (329.48858453024934, 290.1511266046432, 0.037106495159182185, 0.9430402849426585),
}
KNOWN_RMS = (0.0002027456340109754, 0.00010231034501867524)     # check-results.txt:5-6
KNOWN_256 = (4406.5104552251505, 3592.0207507163714, 0.007360143442235456, 0.9899654270279202)  # :7
RTOL = 1e-10


def relerr(a, b):
    return abs(a - b) / abs(b)


def test_time_refinement_known_answers_fp64():
    """checks.jl:16-25 on the GPU: three time steps to t = 10 at 64^2."""
    c0, phi = fields.initial_fields(64, radius=16.0)
    finals = []
    for dt in (0.01, 0.005, 0.0025):
        c, h = esc.run_simulation(c0, phi, dt=dt, steps=round(10 / dt))
        e0, e1, lo, hi = KNOWN_64[dt]
        assert np.max(np.abs(h[:, 1] - c0.mean())) < 1e-12          # checks.jl:19
        assert np.max(np.diff(h[:, 2])) < 1e-8                       # checks.jl:20
        assert relerr(h[0, 2], e0) <= 1e-13
        assert relerr(h[-1, 2], e1) <= RTOL, (dt, h[-1, 2])
        assert relerr(c.min(), lo) <= RTOL and relerr(c.max(), hi) <= RTOL, (dt, c.min(), c.max())
        finals.append(c)
    r1 = np.sqrt(np.mean((finals[0] - finals[1]) ** 2))
    r2 = np.sqrt(np.mean((finals[1] - finals[2]) ** 2))
    assert relerr(r1, KNOWN_RMS[0]) <= 1e-9 and relerr(r2, KNOWN_RMS[1]) <= 1e-9, (r1, r2)


def test_default_example_known_answers_fp64():
    """checks.jl:26-30 on the GPU: the default 256^2 example, 1000 steps."""
    c0, phi = fields.initial_fields(256)
    c, h = esc.run_simulation(c0, phi, dt=0.01, steps=1000)
    e0, e1, lo, hi = KNOWN_256
    assert np.max(np.abs(h[:, 1] - c0.mean())) < 1e-12
    assert np.max(np.diff(h[:, 2])) < 1e-8
    assert relerr(h[0, 2], e0) <= 1e-13 and relerr(h[-1, 2], e1) <= RTOL, h[-1, 2]
    assert relerr(c.min(), lo) <= RTOL and relerr(c.max(), hi) <= RTOL, (c.min(), c.max())


def test_default_example_known_answers_mixed():
    """The mixed mode on the same example, held to its error bound against the known answers."""
    c0, phi = fields.initial_fields(256)
    c, h = esc.run_simulation(c0, phi, dt=0.01, steps=1000, precision="mixed")
    e0, e1, lo, hi = KNOWN_256
    assert np.max(np.abs(h[:, 1] - c0.mean())) < 1e-12
    # f and f' in FP32 (expanded about fl32(c)): the bulk energy sum carries ~1e-8 relative
    assert relerr(h[0, 2], e0) <= 1e-7 and relerr(h[-1, 2], e1) <= 1e-6, (h[0, 2], h[-1, 2])
    assert abs(c.min() - lo) <= 1e-5 and abs(c.max() - hi) <= 1e-5, (c.min(), c.max())


@pytest.mark.parametrize("name", ["disc16_r4", "disc48_r12", "disc64_r16", "disc96_r24_dt005"])
def test_fp64_matches_golden_fixture(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    p = esc.Parameters(*[float(x) for x in d["params"]])
    c, h = esc.run_simulation(d["c0"], d["phi"], dt=float(d["dt"]), steps=int(d["steps"]), p=p)
    assert np.max(np.abs(c - d["c"])) / np.max(np.abs(d["c"])) <= 1e-12
    scale = np.maximum(np.max(np.abs(d["history"]), axis=0), 1e-300)
    assert np.max(np.abs(h - d["history"]) / scale) <= 1e-12
