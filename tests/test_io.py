"""Host I/O: the reference's result files (core_shell.jl:96-101) and the restart format."""
import os

import numpy as np
import pytest

from esc import io


@pytest.mark.parametrize("x,text", [(0.5, "0.5"), (1.0, "1.0"), (10.0, "10.0"), (100000.0, "100000.0"),
                                    (1e6, "1.0e6"), (1.5e-5, "1.5e-5"), (0.0001, "0.0001"),
                                    (123456.789, "123456.789"), (-2.5e-7, "-2.5e-7"), (4406.51, "4406.51"),
                                    (0.1, "0.1"), (0.0, "0.0"), (-3.0, "-3.0"), (2.0e20, "2.0e20"),
                                    (1.2345e-300, "1.2345e-300")])
def test_julia_style_numbers(x, text):
    assert io.julia_float(x) == text


def test_numbers_round_trip():
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.standard_normal(2000) * 10.0 ** rng.integers(-12, 12, 2000),
                         rng.random(500), -rng.random(500)])
    for x in xs:
        assert float(io.julia_float(x)) == x


def test_result_files_layout(tmp_path):
    rng = np.random.default_rng(1)
    c = rng.random((8, 8))
    phi = rng.random((8, 8))
    hist = rng.random((5, 6))
    io.write_results(str(tmp_path), c, hist, phi)
    assert sorted(os.listdir(tmp_path)) == ["composition.csv", "history.csv", "particle.csv"]
    h = np.loadtxt(tmp_path / "history.csv", delimiter=",")
    assert np.array_equal(h, hist)
    # writedlm row i is the Julia matrix row A[i, :] = fixed x (index 1), i.e. column i of a[y, x]
    rows = np.loadtxt(tmp_path / "composition.csv", delimiter=",")
    assert np.array_equal(rows, c.T)
    assert np.array_equal(io.read_field_csv(str(tmp_path / "composition.csv")), c)
    assert np.array_equal(io.read_field_csv(str(tmp_path / "particle.csv")), phi)


def test_restart_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    c = rng.random((16, 16))
    phi = rng.random((16, 16))
    p = str(tmp_path / "state.esc")
    io.save_restart(p, c, step=1234, dt=0.01, dx=0.5, phi=phi)
    c2, phi2, meta = io.load_restart(p)
    assert np.array_equal(c2, c) and np.array_equal(phi2, phi)
    assert meta == {"step": 1234, "dt": 0.01, "dx": 0.5, "time": 12.34}
    assert os.path.getsize(p) == 64 + 2 * 16 * 16 * 8
    io.save_restart(p, c, step=0, dt=0.01)
    c3, phi3, _ = io.load_restart(p)
    assert np.array_equal(c3, c) and phi3 is None


def test_restart_rejects_bad_files(tmp_path):
    p = tmp_path / "bad.esc"
    p.write_bytes(b"not a restart file at all, really not" * 3)
    with pytest.raises(ValueError):
        io.load_restart(str(p))
    good = tmp_path / "good.esc"
    io.save_restart(str(good), np.zeros((4, 4)), 1, 0.01)
    good.write_bytes(good.read_bytes()[:-8])
    with pytest.raises(ValueError):
        io.load_restart(str(good))


def test_conf3d_round_trip(tmp_path):
    """3-D configuration files: c then phi, raw float64, z contiguous (out_conf.cu:39-43)."""
    rng = np.random.default_rng(3)
    c, phi = rng.random((4, 6, 8)), rng.random((4, 6, 8))
    path = io.write_conf3d(str(tmp_path), 120, c, phi)
    assert os.path.basename(path) == "conf.000000120"
    assert os.path.getsize(path) == 2 * c.size * 8
    raw = np.fromfile(path, dtype="<f8")
    assert raw[1] == c[0, 0, 1] and raw[8] == c[0, 1, 0] and raw[c.size] == phi[0, 0, 0]
    c2, phi2 = io.read_conf3d(path, c.shape)
    assert np.array_equal(c2, c) and np.array_equal(phi2, phi)
    with pytest.raises(ValueError):
        io.read_conf3d(path, (4, 6, 7))
