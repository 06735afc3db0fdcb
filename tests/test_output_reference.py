"""The output and restart files against the reference's own code, compiled for the host from its
sources (oracle/_ref/libvfref_io64.so / libvfref_io32.so: WbWriterVtkXmlBinary.cpp and
RestartObject.cpp, built by `make -C oracle ref` where the reference tree is).

* FileWriter's oct files, the parallel collection and the time-series collection written by
  virtualfluids_b200.output are byte-identical to the reference writer's for the same arrays.
* Restart files: what save_restart writes, BinaryRestartObject::deserialize_internal reads back
  exactly, and what the reference's serialize_internal writes, load_restart reads back exactly
  (FP64 and FP32, several levels).
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from virtualfluids_b200 import ListGrid
from virtualfluids_b200 import _native as N
from virtualfluids_b200.output import (FileWriter, level_octs, load_restart, save_restart, write_pvd, write_pvtu,
                                       write_vtu_octs)

REF = Path(__file__).resolve().parent.parent / "oracle" / "_ref"


def _lib(bits):
    p = REF / f"libvfref_io{bits}.so"
    if not p.exists():
        pytest.skip("the reference's writer and restart object are not built here (make -C oracle ref)")
    L = C.CDLL(str(p))
    P, i, u = C.c_void_p, C.c_int, C.c_uint
    L.refio_write_octs.argtypes = [C.c_char_p, i, P, i, P, i, P, P, C.c_char_p, i]
    L.refio_write_parallel_file.argtypes = [C.c_char_p, i, P, i, P, C.c_char_p, i]
    L.refio_write_time_series.argtypes = [C.c_char_p, i, P, P, P, i, C.c_char_p, i]
    L.refio_restart_write.argtypes = [C.c_char_p, i, P, P]
    L.refio_restart_read.argtypes = [C.c_char_p, i, P, P, C.c_int64]
    assert L.refio_real_bytes() == bits // 8
    return L


def _strings(names):
    arr = (C.c_char_p * len(names))(*[n.encode() for n in names])
    return arr


def _cavity_level(n=9, seed=3):
    g = ListGrid(n, n + 1, n - 1)
    for s in ("PX", "MX", "PY", "MY", "MZ"):
        g.add_side(s, "noslip")
    g.add_side("PZ", "velocity", velocity=(0.05, 0.0, 0.0))
    rng = np.random.default_rng(seed)
    m = g.number_of_nodes
    return g, {k: rng.normal(scale=1e-2, size=m) for k in ("rho", "vx", "vy", "vz", "pressure")}


def test_oct_file_is_byte_identical_to_the_reference_writer(tmp_path):
    L = _lib(64)
    rng = np.random.default_rng(5)
    n, m = 40, 7
    pts = rng.normal(size=(n, 3)).astype(np.float32)
    cells = rng.integers(0, n, size=(m, 8)).astype(np.int32)
    fields = {"press": rng.normal(size=n), "rho": rng.normal(size=n), "geo": np.full(n, 19.0)}
    mine = write_vtu_octs(tmp_path / "mine", pts, cells, fields)
    data = np.ascontiguousarray(np.stack(list(fields.values())))
    out = C.create_string_buffer(4096)
    L.refio_write_octs(str(tmp_path / "ref").encode(), n, pts.ctypes.data_as(C.c_void_p), m,
                       np.ascontiguousarray(cells).ctypes.data_as(C.c_void_p), len(fields),
                       C.cast(_strings(list(fields)), C.c_void_p), data.ctypes.data_as(C.c_void_p), out, 4096)
    assert out.value.decode().endswith("ref.bin.vtu") and mine.endswith("mine.bin.vtu")
    assert Path(mine).read_bytes() == Path(out.value.decode()).read_bytes()


@pytest.mark.parametrize("periodic", [False, True])
def test_level_files_match_the_reference_writer(tmp_path, periodic):
    """A level as FileWriter writes it: fluid nodes and their octs (no cells through walls or across
    a periodic wrap), the collection file of the time step and the time series."""
    L = _lib(64)
    if periodic:
        g = ListGrid(6, 5, 4, periodic=(True, True, False))
        g.add_side("MZ", "noslip")
        g.add_side("PZ", "noslip")
        rng = np.random.default_rng(9)
        fields = {k: rng.normal(scale=1e-2, size=g.number_of_nodes) for k in ("rho", "vx", "vy", "vz", "pressure")}
    else:
        g, fields = _cavity_level()
    level = dict(coords=g.coords.astype(np.float64), spacing=1.0, geo=g.geo, neighbor=g.neighbor, **fields)
    w = FileWriter(tmp_path / "mine", density_ratio=1.2, velocity_ratio=0.7)
    files = w.write_timestep(0, [level])
    files += w.write_timestep(10, [level], last=True)
    part = Path(files[0])
    assert part.name == "mine_bin_lev_0_ID_0_Part_1_t_0.vtk.bin.vtu"

    # the same part through the reference writer, from the arrays FileWriter::writeUnstructuredGridLT forms
    n = g.number_of_nodes
    fl = np.nonzero(g.geo == N.GEO_FLUID)[0]
    pts = np.zeros((n, 3), dtype=np.float32)
    pts[fl] = g.coords[:, fl].T.astype(np.float32)
    data = np.zeros((6, n))
    data[0, fl] = fields["pressure"][fl] / 3.0 * 1.2 * 0.7 * 0.7
    data[1, fl] = fields["rho"][fl] / 3.0 * 1.2 * 0.7 * 0.7
    for r, k in ((2, "vx"), (3, "vy"), (4, "vz")):
        data[r, fl] = fields[k][fl] * 0.7
    data[5, fl] = N.GEO_FLUID
    cells = np.ascontiguousarray(level_octs(g.geo, g.neighbor, g.coords, 1.0, 0, n), dtype=np.int32)
    assert 0 < len(cells) < len(fl)
    # the oct selection node by node, as writeUnstructuredGridLT and WriterUtilities spell it
    nbx, nby, nbz = g.neighbor
    loop = []
    for pos in range(n):
        if g.geo[pos] != N.GEO_FLUID:
            continue
        o = [pos, nbx[pos]]
        o += [nby[o[1]], nby[pos], nbz[pos], nbz[o[1]]]
        o += [nbz[o[2]], nbz[o[3]]]
        if np.sqrt(((g.coords[:, o[6]].astype(float) - g.coords[:, o[0]]) ** 2).sum()) > 1.01 * np.sqrt(3.0):
            continue
        if all(g.geo[i] == N.GEO_FLUID for i in o) and not any(i > n for i in o):
            loop.append(o)
    assert np.array_equal(cells, np.array(loop, dtype=np.int32))
    out = C.create_string_buffer(4096)
    names = list(FileWriter.NODE_DATA)
    L.refio_write_octs(str(tmp_path / "ref_part").encode(), n, pts.ctypes.data_as(C.c_void_p), len(cells),
                       cells.ctypes.data_as(C.c_void_p), 6, C.cast(_strings(names), C.c_void_p),
                       np.ascontiguousarray(data).ctypes.data_as(C.c_void_p), out, 4096)
    assert part.read_bytes() == Path(out.value.decode()).read_bytes()

    pvtu = [f for f in files if f.endswith("_t_10.vtk.pvtu")][0]
    pieces = ["mine_bin_lev_0_ID_0_Part_1_t_10.vtk.bin.vtu"]
    L.refio_write_parallel_file(str(tmp_path / "ref_bin_ID_0_t_10.vtk").encode(), 1, C.cast(_strings(pieces), C.c_void_p),
                                6, C.cast(_strings(names), C.c_void_p), out, 4096)
    assert Path(pvtu).read_bytes() == Path(out.value.decode()).read_bytes()

    pvd = [f for f in files if f.endswith(".pvd")][0]
    steps = np.array([0, 10], dtype=np.uint32)
    counts = np.array([1, 1], dtype=np.int32)
    series = ["mine_bin_lev_0_ID_0_Part_1_t_0.vtk.bin.vtu", "mine_bin_lev_0_ID_0_Part_1_t_10.vtk.bin.vtu"]
    L.refio_write_time_series(str(tmp_path / "ref_series").encode(), 2, steps.ctypes.data_as(C.c_void_p),
                              counts.ctypes.data_as(C.c_void_p), C.cast(_strings(series), C.c_void_p), 0, out, 4096)
    assert Path(pvd).read_bytes() == Path(out.value.decode()).read_bytes()


def test_collection_files_for_many_steps_and_groups(tmp_path):
    L = _lib(64)
    out = C.create_string_buffer(4096)
    series = {0: ["a0.vtu", "b0.vtu"], 250: ["a1.vtu"], 1000000: ["a2.vtu", "b2.vtu", "c2.vtu"]}
    for groups in (False, True):
        mine = write_pvd(tmp_path / f"mine{groups}", series, separate_groups=groups)
        files = [f for k in sorted(series) for f in series[k]]
        steps = np.array(sorted(series), dtype=np.uint32)
        counts = np.array([len(series[k]) for k in sorted(series)], dtype=np.int32)
        L.refio_write_time_series(str(tmp_path / f"ref{groups}").encode(), len(steps), steps.ctypes.data_as(C.c_void_p),
                                  counts.ctypes.data_as(C.c_void_p), C.cast(_strings(files), C.c_void_p), int(groups),
                                  out, 4096)
        assert Path(mine).read_bytes() == Path(out.value.decode()).read_bytes()
    mine = write_pvtu(tmp_path / "p", ["x.vtu", "y.vtu"], ["press", "rho"])
    L.refio_write_parallel_file(str(tmp_path / "q").encode(), 2, C.cast(_strings(["x.vtu", "y.vtu"]), C.c_void_p), 2,
                                C.cast(_strings(["press", "rho"]), C.c_void_p), out, 4096)
    assert Path(mine).read_bytes() == Path(out.value.decode()).read_bytes()


@pytest.mark.parametrize("bits", [64, 32])
def test_restart_files_cross_read_with_the_reference(tmp_path, bits):
    L = _lib(bits)
    dt = np.float64 if bits == 64 else np.float32
    rng = np.random.default_rng(bits)
    levels = [rng.normal(size=27 * k).astype(dt) for k in (11, 5, 19)]
    # library -> reference
    save_restart(tmp_path / "mine", levels)
    sizes = np.zeros(3, dtype=np.int64)
    back = [np.zeros(27 * 19, dtype=dt) for _ in range(3)]
    ptrs = (C.c_void_p * 3)(*[b.ctypes.data for b in back])
    assert L.refio_restart_read(str(tmp_path / "mine").encode(), 3, sizes.ctypes.data_as(C.c_void_p),
                                C.cast(ptrs, C.c_void_p), 27 * 19) == 3
    for a, b, n in zip(levels, back, sizes):
        assert n == a.size and np.array_equal(a, b[:n])
    # reference -> library
    src = (C.c_void_p * 3)(*[a.ctypes.data for a in levels])
    sz = np.array([a.size for a in levels], dtype=np.int64)
    L.refio_restart_write(str(tmp_path / "ref").encode(), 3, sz.ctypes.data_as(C.c_void_p), C.cast(src, C.c_void_p))
    got = load_restart(tmp_path / "ref", [dt] * 3)
    for a, b in zip(levels, got):
        assert np.array_equal(a, b)
    assert (tmp_path / "ref.bin").read_bytes() == (tmp_path / "mine.bin").read_bytes()
