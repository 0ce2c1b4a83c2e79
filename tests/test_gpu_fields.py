"""Device field generation (esc_particle_device / esc_noise_device) against the host mirrors."""
import numpy as np
import pytest

import esc
from esc import fields

pytestmark = pytest.mark.gpu

CASES = [("disc", [40.0]), ("band", [-20.0, 25.0]), ("ellipse", [50.0, 30.0]), ("annulus", [20.0, 45.0]),
         ("squircle", [35.0]), ("elliptic_shell", [55.0, 40.0, 15.0]), ("elliptic_hole", [50.0, 30.0, 18.0])]


@pytest.mark.parametrize("shape,params", CASES)
def test_particle_shapes(shape, params):
    import torch
    n = 128
    d = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    esc.particle_device(shape, n, d.data_ptr(), params, width=2.5, spacing=0.9)
    torch.cuda.synchronize()
    host = fields.particle(shape, n, params, width=2.5, spacing=0.9)
    assert np.max(np.abs(d.cpu().numpy() - host)) <= 1e-14


def test_noise_whole_field_and_interior():
    import torch
    n = 96
    c = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    esc.noise_device(n, c.data_ptr(), seed=12345)
    torch.cuda.synchronize()
    assert np.max(np.abs(c.cpu().numpy() - fields.counter_noise(n, 12345))) <= 2e-16
    phi = torch.from_numpy(fields.particle("disc", n, [30.0])).cuda()
    esc.noise_device(n, c.data_ptr(), seed=99, phi_ptr=phi.data_ptr(), mean=0.4, amplitude=0.02)
    torch.cuda.synchronize()
    host = fields.counter_noise(n, 99, phi.cpu().numpy(), mean=0.4, amplitude=0.02)
    assert np.max(np.abs(c.cpu().numpy() - host)) <= 1e-15


def test_bad_arguments_rejected():
    import torch
    d = torch.zeros((8, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(esc.EscError):
        esc.particle_device("ellipse", 8, d.data_ptr(), [0.0, 1.0])
    with pytest.raises(esc.EscError):
        esc.particle_device("disc", 8, d.data_ptr(), [3.0], width=0.0)
