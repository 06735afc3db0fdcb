"""Field output and restart files.

* VTK (legacy binary format, readable by ParaView and VisIt): :func:`write_vtk_image` writes the
  fields of a structured box as STRUCTURED_POINTS; :func:`write_vtk_points` writes the fields of a
  node list (the fluid nodes of a level, at their positions) as an UNSTRUCTURED_GRID of vertices.
  The reference writes the same quantities per level (Output/FileWriter.cpp, UnstructuredGridWriter);
  here the format is VTK's own legacy one, not the reference's writer.
* Restart files in the layout of the reference's BinaryRestartObject (Restart/RestartObject.cpp:
  int32 number of levels, then per level an int32 element count and the population array as
  stored, NaN written as 0): :func:`save_restart` / :func:`load_restart`. For FP64 and FP32 storage
  the file is the one the reference writes for a level of the same layout; 16-bit storage writes its
  2-byte values the same way. The parity is not in the file (the reference derives it from the time
  step): a level restarted at time step t is even when t is even, finer levels are even at every
  coarse step.
"""
from __future__ import annotations

import struct

import numpy as np


def _header(f, title):
    f.write(b"# vtk DataFile Version 3.0\n")
    f.write((title.replace("\n", " ")[:255] + "\n").encode())
    f.write(b"BINARY\n")


def _point_data(f, n, fields):
    f.write(f"POINT_DATA {n}\n".encode())
    for name, arr in fields.items():
        a = np.asarray(arr, dtype=np.float64)
        if a.ndim == 2:
            if a.shape != (3, n):
                raise ValueError(f"vector field {name} must have shape (3, {n})")
            f.write(f"VECTORS {name} double\n".encode())
            f.write(np.ascontiguousarray(a.T, dtype=">f8").tobytes())
        else:
            if a.size != n:
                raise ValueError(f"field {name} must have {n} values")
            f.write(f"SCALARS {name} double 1\nLOOKUP_TABLE default\n".encode())
            f.write(np.ascontiguousarray(a.reshape(-1), dtype=">f8").tobytes())
        f.write(b"\n")


def write_vtk_image(path, shape, fields, origin=(0.0, 0.0, 0.0), spacing=1.0, title="virtualfluids_b200 box"):
    """fields: name -> array of nx*ny*nz values (x fastest) or (3, nx*ny*nz) for a vector."""
    nx, ny, nz = (int(v) for v in shape)
    with open(path, "wb") as f:
        _header(f, title)
        f.write(b"DATASET STRUCTURED_POINTS\n")
        f.write(f"DIMENSIONS {nx} {ny} {nz}\n".encode())
        f.write("ORIGIN {} {} {}\n".format(*(repr(float(o)) for o in origin)).encode())
        f.write(f"SPACING {float(spacing)!r} {float(spacing)!r} {float(spacing)!r}\n".encode())
        _point_data(f, nx * ny * nz, fields)


def write_vtk_points(path, points, fields, title="virtualfluids_b200 level"):
    """points: (3, n) positions; fields: name -> n values or (3, n) for a vector."""
    p = np.asarray(points, dtype=np.float64)
    n = p.shape[1]
    with open(path, "wb") as f:
        _header(f, title)
        f.write(b"DATASET UNSTRUCTURED_GRID\n")
        f.write(f"POINTS {n} double\n".encode())
        f.write(np.ascontiguousarray(p.T, dtype=">f8").tobytes())
        f.write(f"\nCELLS {n} {2 * n}\n".encode())
        cells = np.empty((n, 2), dtype=">i4")
        cells[:, 0] = 1
        cells[:, 1] = np.arange(n)
        f.write(cells.tobytes())
        f.write(f"\nCELL_TYPES {n}\n".encode())
        f.write(np.ones(n, dtype=">i4").tobytes())     # VTK_VERTEX
        f.write(b"\n")
        _point_data(f, n, fields)


def read_vtk(path):
    """Reads back the legacy binary files these writers produce: dict with 'dataset', 'points'
    or 'dimensions'/'origin'/'spacing', and the point fields."""
    with open(path, "rb") as f:
        data = f.read()
    pos = 0

    def line():
        nonlocal pos
        end = data.index(b"\n", pos)
        out = data[pos:end].decode()
        pos = end + 1
        return out

    def block(count, dtype):
        nonlocal pos
        nbytes = count * np.dtype(dtype).itemsize
        arr = np.frombuffer(data, dtype=dtype, count=count, offset=pos).astype(np.float64 if "f" in dtype else np.int64)
        pos += nbytes
        return arr

    out = {}
    line(), line()
    if line().strip() != "BINARY":
        raise ValueError("not a binary legacy VTK file")
    out["dataset"] = line().split()[1]
    n = None
    while pos < len(data):
        words = line().split()
        if not words:
            continue
        key = words[0]
        if key == "DIMENSIONS":
            out["dimensions"] = tuple(int(w) for w in words[1:4])
        elif key == "ORIGIN":
            out["origin"] = tuple(float(w) for w in words[1:4])
        elif key == "SPACING":
            out["spacing"] = tuple(float(w) for w in words[1:4])
        elif key == "POINTS":
            m = int(words[1])
            out["points"] = block(3 * m, ">f8").reshape(m, 3).T
        elif key == "CELLS":
            block(int(words[2]), ">i4")
        elif key == "CELL_TYPES":
            block(int(words[1]), ">i4")
        elif key == "POINT_DATA":
            n = int(words[1])
        elif key == "SCALARS":
            line()                                      # LOOKUP_TABLE
            out[words[1]] = block(n, ">f8")
        elif key == "VECTORS":
            out[words[1]] = block(3 * n, ">f8").reshape(n, 3).T
    return out


def save_restart(path, levels):
    """levels: population arrays (one per level, as stored). Writes `path` + ".bin"."""
    with open(str(path) + ".bin", "wb") as f:
        f.write(struct.pack("<i", len(levels)))
        for a in levels:
            a = np.ascontiguousarray(a).reshape(-1)
            if a.size >= 2 ** 31:
                raise ValueError("a level holds more values than the format's int32 count")
            if a.dtype.kind == "f":
                a = np.where(np.isnan(a), a.dtype.type(0), a)
            f.write(struct.pack("<i", a.size))
            f.write(a.tobytes())


def load_restart(path, dtypes):
    """The population arrays of `path` + ".bin", one per level, with the element types given
    (numpy dtypes, one per level; 16-bit storage as np.uint16 raw values)."""
    with open(str(path) + ".bin", "rb") as f:
        data = f.read()
    (levels,) = struct.unpack_from("<i", data, 0)
    if levels != len(dtypes):
        raise ValueError(f"the file holds {levels} levels, {len(dtypes)} expected")
    pos, out = 4, []
    for dt in dtypes:
        (size,) = struct.unpack_from("<i", data, pos)
        pos += 4
        dt = np.dtype(dt)
        out.append(np.frombuffer(data, dtype=dt, count=size, offset=pos).copy())
        pos += size * dt.itemsize
    if pos != len(data):
        raise ValueError("trailing bytes after the last level")
    return out
