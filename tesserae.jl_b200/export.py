"""VTK and PLY output of particles and grids (Tesserae.jl src/IO/export.jl).

The reference writes through WriteVTK.jl; this module writes the same VTK XML
datasets itself (no third-party writer is available here):

* particles -> an UnstructuredGrid (.vtu) of VTK_VERTEX cells, one per particle
  (export.jl:49-54);
* a Cartesian mesh -> a StructuredGrid (.vts) of its nodes (export.jl:55-57);
* several datasets of one time -> a multiblock file (.vtm) (`openvtm`);
* a time series -> a ParaView collection (.pvd) (`openpvd`, `pvd[t] = vtm`).

As in the reference, coordinates and every Float64 field are written as Float32
(export.jl:71-78, 103-106), 2D points and vectors are padded to 3 components, and
a symmetric tensor is written as the 6 components (xx, yy, zz, xy, yz, zx)
(export.jl:79-85; in 2D the missing components are NaN). Arrays are base64
binary with a UInt64 size header, a form ParaView and VTK readers take.
`write_ply` writes the binary little-endian point cloud of export.jl:116-132.

Data on the device is copied to the host first (the reference's `cpu(...)`).
"""
from __future__ import annotations

import base64
import os
import pathlib
import struct
import xml.etree.ElementTree as ET

import numpy as np

VTK_VERTEX = 1


def _host(a) -> np.ndarray:
    if isinstance(a, np.ndarray):
        return a
    return a.detach().cpu().numpy()


def _points3(x) -> np.ndarray:
    """(dim, n) positions -> (n, 3) Float32."""
    x = _host(x)
    dim, n = x.shape
    out = np.zeros((n, 3), dtype=np.float32)
    out[:, :dim] = x.T.astype(np.float32)
    return out


def vtk_format_field(a, kind: str | None = None) -> np.ndarray:
    """A field as VTK components, (n, k) Float32 (or (n,) for scalars).

    kind: "scalar" (n,), "vector" (dim, n) -> 3 components, "symmetric"
    (nsym, n) in Tensorial order 11,21,31,22,32,33 (2D: 11,21,22) -> 6 components
    (xx, yy, zz, xy, yz, zx), "tensor" (dim*dim, n) column-major -> dim*dim
    components. Without `kind`, a 1-D array is a scalar and a 2-D one a vector.
    """
    a = _host(a)
    if kind is None:
        kind = "scalar" if a.ndim == 1 else "vector"
    if kind == "scalar":
        return a.astype(np.float32)
    if kind == "vector":
        d, n = a.shape
        out = np.zeros((n, 3), dtype=np.float32)
        out[:, :d] = a.T.astype(np.float32)
        return out
    if kind == "symmetric":
        k, n = a.shape
        out = np.empty((n, 6), dtype=np.float32)
        if k == 6:   # 11 21 31 22 32 33 -> xx yy zz xy yz zx
            order = (0, 3, 5, 1, 4, 2)
            for j, i in enumerate(order):
                out[:, j] = a[i].astype(np.float32)
        elif k == 3:  # 2D: 11 21 22 -> xx yy NaN xy NaN NaN (export.jl:79-81)
            out[:, 0] = a[0]
            out[:, 1] = a[2]
            out[:, 2] = np.nan
            out[:, 3] = a[1]
            out[:, 4] = np.nan
            out[:, 5] = np.nan
        else:
            raise ValueError("symmetric tensor needs 3 (2D) or 6 (3D) components")
        return out
    if kind == "tensor":
        k, n = a.shape
        return a.T.astype(np.float32).reshape(n, k)
    raise ValueError(f"unknown field kind {kind!r}")


def _data_array(parent: ET.Element, name: str | None, arr: np.ndarray):
    arr = np.ascontiguousarray(arr)
    ncomp = 1 if arr.ndim == 1 else arr.shape[1]
    type_name = {np.dtype(np.float32): "Float32", np.dtype(np.float64): "Float64",
                 np.dtype(np.int64): "Int64", np.dtype(np.uint8): "UInt8", np.dtype(np.int32): "Int32"}[arr.dtype]
    attrs = {"type": type_name, "NumberOfComponents": str(ncomp), "format": "binary"}
    if name is not None:
        attrs["Name"] = name
    el = ET.SubElement(parent, "DataArray", attrs)
    raw = arr.astype(arr.dtype.newbyteorder("<"), copy=False).tobytes()
    el.text = base64.b64encode(struct.pack("<Q", len(raw)) + raw).decode("ascii")
    return el


def _vtkfile(kind: str) -> tuple[ET.Element, ET.Element]:
    root = ET.Element("VTKFile", {"type": kind, "version": "1.0", "byte_order": "LittleEndian",
                                  "header_type": "UInt64"})
    return root, ET.SubElement(root, kind)


def _write(root: ET.Element, path: pathlib.Path):
    ET.ElementTree(root).write(path, xml_declaration=True, encoding="utf-8")


def write_particles(path, x, fields: dict | None = None, kinds: dict | None = None) -> pathlib.Path:
    """Particles as a .vtu of VTK_VERTEX cells (export.jl:49-54, openvtk).
    `x` is (dim, n); `fields` maps names to arrays (see vtk_format_field);
    `kinds` gives a field's kind where it is not a plain scalar or vector."""
    path = pathlib.Path(path).with_suffix(".vtu")
    pts = _points3(x)
    n = pts.shape[0]
    root, grid = _vtkfile("UnstructuredGrid")
    piece = ET.SubElement(grid, "Piece", {"NumberOfPoints": str(n), "NumberOfCells": str(n)})
    pd = ET.SubElement(piece, "PointData")
    for name, a in (fields or {}).items():
        _data_array(pd, name, vtk_format_field(a, (kinds or {}).get(name)))
    _data_array(ET.SubElement(piece, "Points"), "Points", pts)
    cells = ET.SubElement(piece, "Cells")
    _data_array(cells, "connectivity", np.arange(n, dtype=np.int64))
    _data_array(cells, "offsets", np.arange(1, n + 1, dtype=np.int64))
    _data_array(cells, "types", np.full(n, VTK_VERTEX, dtype=np.uint8))
    _write(root, path)
    return path


def write_grid(path, mesh, fields: dict | None = None, kinds: dict | None = None) -> pathlib.Path:
    """A Cartesian mesh's nodes as a .vts structured grid (export.jl:55-57) with
    node fields (arrays of prod(n_nodes) entries per component, column-major
    node order as the grid's)."""
    path = pathlib.Path(path).with_suffix(".vts")
    dim = mesh.dim
    nn = list(mesh.n_nodes) + [1] * (3 - dim)
    axes = [mesh.xmin[d] + np.arange(mesh.n_nodes[d]) * mesh.h for d in range(dim)] + [np.zeros(1)] * (3 - dim)
    X = np.meshgrid(*axes, indexing="ij")
    pts = np.stack([g.reshape(-1, order="F") for g in X], axis=1).astype(np.float32)
    extent = " ".join(f"0 {k - 1}" for k in nn)
    root, grid = _vtkfile("StructuredGrid")
    grid.set("WholeExtent", extent)
    piece = ET.SubElement(grid, "Piece", {"Extent": extent})
    pd = ET.SubElement(piece, "PointData")
    for name, a in (fields or {}).items():
        _data_array(pd, name, vtk_format_field(a, (kinds or {}).get(name)))
    _data_array(ET.SubElement(piece, "Points"), "Points", pts)
    _write(root, path)
    return path


def write_multiblock(path, files: list) -> pathlib.Path:
    """A .vtm referring to datasets written beside it (openvtm)."""
    path = pathlib.Path(path).with_suffix(".vtm")
    root, mb = _vtkfile("vtkMultiBlockDataSet")
    for i, f in enumerate(files):
        ET.SubElement(mb, "DataSet", {"index": str(i), "file": os.path.relpath(f, path.parent)})
    _write(root, path)
    return path


class Collection:
    """A ParaView collection (.pvd) of time steps (openpvd; `pvd[t] = vtm`)."""

    def __init__(self, path):
        self.path = pathlib.Path(path).with_suffix(".pvd")
        self.entries: list[tuple[float, pathlib.Path]] = []

    def __setitem__(self, t: float, file):
        self.entries.append((float(t), pathlib.Path(file)))

    def save(self) -> pathlib.Path:
        root = ET.Element("VTKFile", {"type": "Collection", "version": "1.0", "byte_order": "LittleEndian"})
        col = ET.SubElement(root, "Collection")
        for t, f in self.entries:
            ET.SubElement(col, "DataSet", {"timestep": repr(t), "part": "0",
                                            "file": os.path.relpath(f, self.path.parent)})
        _write(root, self.path)
        return self.path

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.save()


def write_ply(name, x) -> pathlib.Path:
    """Binary little-endian PLY of the points (export.jl:116-132): the header
    lines, then x, y, z as Float32 per point (2D padded with z = 0)."""
    path = pathlib.Path(f"{name}.ply")
    pts = _points3(x)
    header = ("ply\nformat binary_little_endian 1.0\n"
              f"element vertex {pts.shape[0]}\nproperty float x\nproperty float y\nproperty float z\nend_header\n")
    with open(path, "wb") as f:
        f.write(header.encode("ascii"))
        f.write(pts.astype("<f4").tobytes())
    return path


def read_data_arrays(path) -> dict:
    """The arrays of a file written here, by name (Points, PointData fields,
    cell arrays), decoded to numpy: for checking output."""
    out = {}
    for el in ET.parse(path).getroot().iter("DataArray"):
        raw = base64.b64decode(el.text)
        (nbytes,) = struct.unpack("<Q", raw[:8])
        dt = {"Float32": "<f4", "Float64": "<f8", "Int64": "<i8", "UInt8": "u1", "Int32": "<i4"}[el.get("type")]
        a = np.frombuffer(raw[8:8 + nbytes], dtype=dt)
        k = int(el.get("NumberOfComponents", "1"))
        out[el.get("Name")] = a.reshape(-1, k) if k > 1 else a
    return out
