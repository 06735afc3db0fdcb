"""Field output and restart files.

* The reference's output files (Output/FileWriter.cpp): :class:`FileWriter` writes each level of a
  time step as VTK XML unstructured grids of hexahedral cells ("octs") with FP64 point data in raw
  appended binary (the layout of the reference's WbWriterVtkXmlBinary::writeOctsWithNodeData,
  ``*.bin.vtu``), split into parts of at most 30 million nodes, plus the parallel collection file
  of the time step (``*.pvtu``) and the time-series collection (``*.pvd``). The same arrays give the
  same bytes as the reference's writer (checked against it, compiled from its sources, in
  tests/test_output.py).
* VTK legacy binary files (readable by ParaView and VisIt): :func:`write_vtk_image` writes the
  fields of a structured box as STRUCTURED_POINTS; :func:`write_vtk_points` writes the fields of a
  node list as an UNSTRUCTURED_GRID of vertices.
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


# Output/FilePartCalculator.h:53: at most this many nodes per part file
VTK_NODES_PER_PART = 30_000_000
# VTK_VOXEL, the cell type of the oct files
_VTK_VOXEL = 11


def write_vtu_octs(filename, points, cells, fields):
    """An unstructured grid of octs with FP64 point data: writes ``filename + ".bin.vtu"`` and
    returns that name (WbWriterVtkXmlBinary::writeOctsWithNodeData, basics/writer/
    WbWriterVtkXmlBinary.cpp:1306-1422: XML header with appended-data offsets, then raw little-endian
    blocks each led by its int32 byte count).

    points: (n, 3) positions (stored as float32); cells: (m, 8) node indices of each oct in the order
    base, +x, +x+y, +y, +z, +x+z, +x+y+z, +y+z (written in VTK voxel order); fields: ordered mapping
    name -> n values (stored as float64)."""
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float32).reshape(-1, 3))
    octs = np.asarray(cells, dtype=np.int32).reshape(-1, 8)
    n, m = pts.shape[0], octs.shape[0]
    names = list(fields)
    b_points, b_conn, b_off, b_types, b_scalar = 12 * n, 32 * m, 4 * m, m, 8 * n
    offs = [0]
    for size in (b_points, b_conn, b_off, b_types):
        offs.append(offs[-1] + 4 + size)
    data_offs = [offs[4] + k * (4 + b_scalar) for k in range(len(names))]
    head = ['<?xml version="2.0"?>\n',
            '<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian" >\n',
            "   <UnstructuredGrid>\n",
            f'      <Piece NumberOfPoints="{n}" NumberOfCells="{m}">\n',
            "         <Points>\n",
            f'            <DataArray type="Float32" NumberOfComponents="3" format="appended" offset="{offs[0]}"  />\n',
            "         </Points>\n",
            "         <Cells>\n",
            f'            <DataArray type="Int32" Name="connectivity" format="appended" offset="{offs[1]}" />\n',
            f'            <DataArray type="Int32" Name="offsets" format="appended" offset="{offs[2]}" />\n',
            f'            <DataArray type="UInt8" Name="types" format="appended" offset="{offs[3]}" />\n ',
            "         </Cells>\n",
            "         <PointData>\n"]
    head += [f'            <DataArray type="Float64" Name="{name}" format="appended" offset="{o}" /> \n'
             for name, o in zip(names, data_offs)]
    head += ["         </PointData>\n", "      </Piece>\n", "   </UnstructuredGrid>\n",
             '   <AppendedData encoding="raw">\n', "_"]
    conn = np.ascontiguousarray(octs[:, [0, 1, 3, 2, 4, 5, 7, 6]], dtype="<i4")
    out_name = str(filename) + ".bin.vtu"
    with open(out_name, "wb") as f:
        f.write("".join(head).encode())
        f.write(struct.pack("<i", b_points))
        f.write(pts.astype("<f4").tobytes())
        f.write(struct.pack("<i", b_conn))
        f.write(conn.tobytes())
        f.write(struct.pack("<i", b_off))
        f.write((8 * np.arange(1, m + 1, dtype="<i4")).tobytes())
        f.write(struct.pack("<i", b_types))
        f.write(np.full(m, _VTK_VOXEL, dtype=np.uint8).tobytes())
        for name in names:
            a = np.asarray(fields[name], dtype="<f8").reshape(-1)
            if a.size != n:
                raise ValueError(f"field {name} must have {n} values")
            f.write(struct.pack("<i", b_scalar))
            f.write(a.tobytes())
        f.write(b"\n</AppendedData>\n</VTKFile>\n")
    return out_name


def write_pvtu(filename, pieces, point_data_names):
    """The parallel collection of one time step (WbWriterVtkXmlBinary::writeParallelFile,
    WbWriterVtkXmlBinary.cpp:141-176, without cell data): ``filename + ".pvtu"``."""
    lines = ['<?xml version="1.0"?>', '<VTKFile type="PUnstructuredGrid" version="0.1" byte_order="LittleEndian">',
             '  <PUnstructuredGrid GhostLevel="1">', "    <PPointData>"]
    lines += [f'      <PDataArray type="Float64" Name="{n}"/>' for n in point_data_names]
    lines += ["    </PPointData>", "    <PPoints>", '      <PDataArray type="Float32" NumberOfComponents="3"/>',
              "    </PPoints>"]
    lines += [f'    <Piece Source="{p}"/>' for p in pieces]
    lines += ["  </PUnstructuredGrid>", "</VTKFile>"]
    out_name = str(filename) + ".pvtu"
    with open(out_name, "wb") as f:
        f.write(("\n".join(lines) + "\n").encode())
    return out_name


def _ostream_double(x):
    """A double as std::ostream writes it by default (six significant digits, %g)."""
    return "%g" % float(x)


def write_pvd(filename, series, separate_groups=False):
    """The time-series collection (WbWriterVtkXmlBinary::writeCollectionForTimeSeries,
    WbWriterVtkXmlBinary.cpp:58-99): ``filename + ".pvd"``; series maps time step -> file names."""
    lines = ['<VTKFile type="Collection" version="0.1" byte_order="LittleEndian" >', "   <Collection>"]
    for step in sorted(series):
        group = part = 0
        for name in series[step]:
            lines.append(f'       <DataSet timestep="{_ostream_double(step)}" group="{group}" part="{part}" '
                         f'file="{name}"/>')
            if separate_groups:
                group += 1
            else:
                part += 1
    out_name = str(filename) + ".pvd"
    with open(out_name, "wb") as f:
        f.write(("\n".join(lines) + "\n   </Collection>\n</VTKFile>").encode())
    return out_name


def level_octs(geo, neighbor, coords, spacing, start, end, fluid_code=19):
    """The octs of the nodes [start, end) of a level as FileWriter::writeUnstructuredGridLT forms
    them (FileWriter.cpp:267-311, WriterUtilities.cpp): from every fluid node, its +x, +x+y, +y,
    +z, +x+z, +x+y+z, +y+z neighbours through neighborX/Y/Z; dropped when any of the eight is not
    fluid, lies beyond `end`, or the cell's diagonal is longer than 1.01 sqrt(3) spacings (a cell
    across a periodic wrap). Returns (m, 8) node indices relative to `start`."""
    nbx, nby, nbz = (np.asarray(a, dtype=np.int64) for a in neighbor)
    geo = np.asarray(geo)
    base = np.arange(start, end, dtype=np.int64)
    base = base[geo[base] == fluid_code]
    i1 = nbx[base]
    i2 = nby[i1]
    i3 = nby[base]
    idx = np.stack([base, i1, i2, i3, nbz[base], nbz[i1], nbz[i2], nbz[i3]], axis=1)
    c = np.asarray(coords, dtype=np.float64)
    d = np.sqrt(((c[:, idx[:, 6]] - c[:, idx[:, 0]]) ** 2).sum(axis=0))
    keep = d <= 1.01 * np.sqrt(3.0 * spacing ** 2)
    keep &= np.all(geo[idx] == fluid_code, axis=1) & np.all(idx <= end, axis=1)
    return idx[keep] - start


class FileWriter:
    """The reference's field output (Output/FileWriter.cpp): per time step, every level in part
    files ``<prefix>_bin_lev_<l>_ID_<id>_Part_<p>_t_<t>.vtk.bin.vtu`` with the point data press,
    rho (both / 3 * densityRatio * velocityRatio^2), vx1, vx2, vx3 (* velocityRatio) and geo of
    every fluid node at its position (non-fluid entries zero), then ``<prefix>_bin_ID_<id>_t_<t>.vtk.pvtu``
    over those parts; after the last time step ``<prefix>_bin_ID_<id>.pvd`` over all of them."""

    NODE_DATA = ("press", "rho", "vx1", "vx2", "vx3", "geo")

    def __init__(self, prefix, process_id=0, density_ratio=1.0, velocity_ratio=1.0):
        self.prefix = str(prefix)
        self.process_id = int(process_id)
        self.density_ratio = float(density_ratio)
        self.velocity_ratio = float(velocity_ratio)
        self.series = {}

    def write_timestep(self, timestep, levels, last=False):
        """levels: per level a dict with coords (3, n), spacing, geo, neighbor (3 arrays) and the
        macroscopic arrays rho, vx, vy, vz, pressure (n values each). Returns the files written."""
        t, pid = int(timestep), self.process_id
        pieces, written = [], []
        for lev, L in enumerate(levels):
            n = len(L["geo"])
            parts = n // VTK_NODES_PER_PART + 1
            for part in range(parts):
                start = part * VTK_NODES_PER_PART
                size = n - start if part == parts - 1 else VTK_NODES_PER_PART
                end = start + size
                name = f"{self.prefix}_bin_lev_{lev}_ID_{pid}_Part_{part + 1}_t_{t}.vtk"
                written.append(self._write_part(name, L, start, end))
                pieces.append(written[-1].replace("\\", "/").rsplit("/", 1)[-1])
        self.series[t] = list(pieces)
        if last:
            written.append(write_pvd(f"{self.prefix}_bin_ID_{pid}", self.series))
        written.append(write_pvtu(f"{self.prefix}_bin_ID_{pid}_t_{t}.vtk", pieces, self.NODE_DATA))
        return written

    def _write_part(self, name, L, start, end):
        geo = np.asarray(L["geo"])
        sel = np.arange(start, end)
        fl = sel[geo[sel] == 19]
        rel = fl - start
        size = end - start
        pts = np.zeros((size, 3), dtype=np.float32)
        pts[rel] = np.asarray(L["coords"], dtype=np.float64)[:, fl].T.astype(np.float32)
        dr, vr = self.density_ratio, self.velocity_ratio
        data = {k: np.zeros(size) for k in self.NODE_DATA}
        data["press"][rel] = np.asarray(L["pressure"], dtype=np.float64)[fl] / 3.0 * dr * vr * vr
        data["rho"][rel] = np.asarray(L["rho"], dtype=np.float64)[fl] / 3.0 * dr * vr * vr
        for key, src in (("vx1", "vx"), ("vx2", "vy"), ("vx3", "vz")):
            data[key][rel] = np.asarray(L[src], dtype=np.float64)[fl] * vr
        data["geo"][rel] = geo[fl].astype(np.float64)
        cells = level_octs(geo, L["neighbor"], L["coords"], float(L["spacing"]), start, end)
        return write_vtu_octs(name, pts, cells, data)


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
