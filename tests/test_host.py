"""Host-side logic of the Python mirror that needs no GPU."""
import numpy as np
import pytest

import esc
from esc import fields
from oracle import core_shell_oracle as orc


def test_field_generators_match_oracle_restatement():
    for n, r, w, s in [(64, 16.0, 4.0, 5749), (96, 30.0, 2.0, 3), (256, 70.0, 4.0, 1)]:
        c, phi = fields.initial_fields(n, radius=r, width=w, seed=s)
        co, phio = orc.initial_fields(n, radius=r, width=w, seed=s)
        assert np.array_equal(c, co) and np.array_equal(phi, phio)
    assert np.array_equal(fields.particle_ellipse(128, 50.0, 30.0, 2.0), orc.particle_ellipse(128, 50.0, 30.0, 2.0))
    assert np.array_equal(fields.whole_field_noise(64, 1), orc.whole_field_noise(64, 1))


def test_initial_fields_properties():
    c, phi = fields.initial_fields(256)                     # core_shell.jl:27-37
    inside = phi >= 0.5
    assert phi[128, 128] > 0.99 and phi[0, 0] < 1e-6        # centred on index n÷2
    assert abs(c[inside].mean() - 0.5) < 1e-15              # interior mean removed
    assert np.all(c[~inside] == 0.5)
    assert np.max(np.abs(c - 0.5)) <= 0.02
    assert np.array_equal(phi, phi.T)


def test_ellipse_axes():
    phi = fields.particle_ellipse(512, a=200.0, b=120.0, width=2.0)
    row = phi[256]                                          # along x (axis 1), semi-axis a
    col = phi[:, 256]                                       # along y, semi-axis b
    assert abs(np.sum(row >= 0.5) - 401) <= 2 and abs(np.sum(col >= 0.5) - 241) <= 2


def test_batch_argument_validation():
    with pytest.raises(ValueError):
        esc.Batch([])
    with pytest.raises(ValueError):
        esc.Batch([np.zeros((8, 4))])
    with pytest.raises(ValueError):
        esc.Batch([np.zeros((8, 8))], spacings=[1.0, 2.0])


def test_field_shape_checks():
    with pytest.raises(ValueError):
        esc._field(np.zeros((8, 9)), 8, "c0")
    a = esc._field(np.zeros((8, 8), dtype=np.float32), 8, "c0")
    assert a.dtype == np.float64 and a.flags.c_contiguous


def test_splitmix_known_answer():
    """The first SplitMix64 output of state 0 is 0xE220A8397B1DCDAF (published test value)."""
    from esc import fields
    u = fields.splitmix_uniform(0, 2)
    assert u[0] == (0xE220A8397B1DCDAF >> 11) / 9007199254740992.0
    assert 0.0 <= u[1] < 1.0


def test_counter_noise_interior_mean_removed():
    from esc import fields
    phi = fields.particle("disc", 64, [20.0])
    c = fields.counter_noise(64, 7, phi)
    inside = phi >= 0.5
    assert abs(c[inside].mean() - 0.5) < 1e-15
    assert np.all(c[~inside] == 0.5)
    assert np.max(np.abs(c - 0.5)) <= 0.02


def test_host_shapes_match_the_disc_and_ellipse_generators():
    from esc import fields
    assert np.array_equal(fields.particle("disc", 32, [10.0], width=4.0), fields.particle_disc(32, 1.0, 10.0, 4.0))
    assert np.array_equal(fields.particle("ellipse", 48, [20.0, 12.0], width=2.0),
                          fields.particle_ellipse(48, 20.0, 12.0, 2.0))
