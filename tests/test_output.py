"""Field output (legacy VTK) and restart files on the host: the writers' files read back to the same
values, and restart files follow the reference's binary restart layout (int32 level count, then
per level an int32 count and the values, NaN stored as 0)."""
import struct

import numpy as np
import pytest

from virtualfluids_b200.output import load_restart, read_vtk, save_restart, write_vtk_image, write_vtk_points


def test_vtk_image_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    shape = (5, 4, 3)
    n = 60
    rho, vel = rng.normal(size=n), rng.normal(size=(3, n))
    p = tmp_path / "box.vtk"
    write_vtk_image(p, shape, {"drho": rho, "velocity": vel}, origin=(1.0, 2.0, 3.0), spacing=0.5)
    back = read_vtk(p)
    assert back["dataset"] == "STRUCTURED_POINTS" and back["dimensions"] == shape
    assert back["origin"] == (1.0, 2.0, 3.0) and back["spacing"] == (0.5, 0.5, 0.5)
    assert np.array_equal(back["drho"], rho) and np.array_equal(back["velocity"], vel)


def test_vtk_points_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    pts, rho, vel = rng.normal(size=(3, 17)), rng.normal(size=17), rng.normal(size=(3, 17))
    p = tmp_path / "level.vtk"
    write_vtk_points(p, pts, {"drho": rho, "velocity": vel})
    back = read_vtk(p)
    assert back["dataset"] == "UNSTRUCTURED_GRID"
    assert np.array_equal(back["points"], pts) and np.array_equal(back["drho"], rho)
    assert np.array_equal(back["velocity"], vel)
    with pytest.raises(ValueError):
        write_vtk_points(p, pts, {"drho": rho[:5]})


def test_restart_layout_and_round_trip(tmp_path):
    a = np.arange(27 * 5, dtype=np.float64) * 0.5
    a[3] = np.nan
    b = np.arange(27 * 2, dtype=np.float32)
    c = np.arange(27, dtype=np.uint16)
    save_restart(tmp_path / "r", [a, b, c])
    raw = (tmp_path / "r.bin").read_bytes()
    assert struct.unpack_from("<ii", raw, 0) == (3, a.size)
    assert struct.unpack_from("<d", raw, 8 + 8 * 3)[0] == 0.0          # NaN written as 0
    back = load_restart(tmp_path / "r", [np.float64, np.float32, np.uint16])
    want = a.copy()
    want[3] = 0.0
    assert np.array_equal(back[0], want) and np.array_equal(back[1], b) and np.array_equal(back[2], c)
    with pytest.raises(ValueError):
        load_restart(tmp_path / "r", [np.float64, np.float32])
    with pytest.raises(ValueError):
        load_restart(tmp_path / "r", [np.float64, np.float64, np.uint16])
