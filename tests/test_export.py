"""VTK / PLY output (src/IO/export.jl): files written for particles and grids
are read back and checked against the arrays they were written from: Float32
coordinates padded to 3D, one VTK_VERTEX cell per particle, symmetric tensors
as (xx, yy, zz, xy, yz, zx) with NaN for the components a 2D tensor lacks, node
coordinates of a CartesianMesh in column-major order, and the multiblock /
collection files naming their datasets."""
import xml.etree.ElementTree as ET

import numpy as np


def test_particles_vtu_3d(tb, tmp_path):
    from tesserae_b200 import export
    sc = tb.scenes.cube3d(scale=8)
    P = sc.particles
    rng = np.random.default_rng(7)
    P.sigma[:] = rng.standard_normal(P.sigma.shape)
    path = export.write_particles(tmp_path / "particles", P.x,
                                  {"velocity": P.v, "volume": P.V, "stress": P.sigma, "F": P.F},
                                  kinds={"stress": "symmetric", "F": "tensor"})
    assert path.suffix == ".vtu"
    a = export.read_data_arrays(path)
    assert a["Points"].dtype == np.float32 and a["Points"].shape == (P.n, 3)
    assert np.array_equal(a["Points"], P.x.T.astype(np.float32))
    assert np.array_equal(a["velocity"], P.v.T.astype(np.float32))
    assert np.array_equal(a["volume"], P.V.astype(np.float32))
    s = P.sigma.astype(np.float32)  # stored 11 21 31 22 32 33
    want = np.stack([s[0], s[3], s[5], s[1], s[4], s[2]], axis=1)
    assert np.array_equal(a["stress"], want)
    assert np.array_equal(a["F"], P.F.T.astype(np.float32))
    assert np.array_equal(a["types"], np.ones(P.n, np.uint8))
    assert np.array_equal(a["connectivity"], np.arange(P.n))
    assert np.array_equal(a["offsets"], np.arange(1, P.n + 1))
    root = ET.parse(path).getroot()
    assert root.get("type") == "UnstructuredGrid"
    piece = root.find("UnstructuredGrid/Piece")
    assert piece.get("NumberOfPoints") == str(P.n) and piece.get("NumberOfCells") == str(P.n)


def test_particles_2d_padding_and_symmetric_nan(tb, tmp_path):
    from tesserae_b200 import export
    P = tb.scenes.readme2d().particles
    P.sigma[:] = np.arange(3)[:, None] + 1.0
    path = export.write_particles(tmp_path / "p2d", P.x, {"v": P.v, "sigma": P.sigma},
                                  kinds={"sigma": "symmetric"})
    a = export.read_data_arrays(path)
    assert np.array_equal(a["Points"][:, :2], P.x.T.astype(np.float32))
    assert np.all(a["Points"][:, 2] == 0) and np.all(a["v"][:, 2] == 0)
    s = a["sigma"]
    assert np.all(s[:, 0] == 1) and np.all(s[:, 1] == 3) and np.all(s[:, 3] == 2)
    assert np.all(np.isnan(s[:, [2, 4, 5]]))


def test_grid_vts(tb, tmp_path):
    from tesserae_b200 import export
    mesh = tb.CartesianMesh(0.5, (0.0, 2.0), (-1.0, 0.5), (1.0, 2.0))
    G = tb.generate_grid(mesh)
    G.m[:] = np.arange(mesh.nnodes)
    G.v[:] = np.arange(3 * mesh.nnodes).reshape(3, -1)
    path = export.write_grid(tmp_path / "grid", mesh, {"mass": G.m, "velocity": G.v})
    root = ET.parse(path).getroot()
    nx, ny, nz = mesh.n_nodes
    assert root.find("StructuredGrid").get("WholeExtent") == f"0 {nx - 1} 0 {ny - 1} 0 {nz - 1}"
    a = export.read_data_arrays(path)
    X = a["Points"]
    # column-major: x varies fastest
    i, j, k = 1, 2, 1
    n = i + nx * (j + ny * k)
    assert np.allclose(X[n], [0.0 + 0.5 * i, -1.0 + 0.5 * j, 1.0 + 0.5 * k])
    assert np.array_equal(a["mass"], G.m.astype(np.float32))
    assert np.array_equal(a["velocity"], G.v.T.astype(np.float32))


def test_multiblock_and_collection(tb, tmp_path):
    from tesserae_b200 import export
    sc = tb.scenes.cube3d(scale=8)
    with export.Collection(tmp_path / "out" / "run") as pvd:
        (tmp_path / "out").mkdir()
        for step, t in enumerate((0.0, 0.5)):
            fp = export.write_particles(tmp_path / "out" / f"particles_{step}", sc.particles.x)
            fg = export.write_grid(tmp_path / "out" / f"grid_{step}", sc.mesh)
            pvd[t] = export.write_multiblock(tmp_path / "out" / f"run_{step}", [fp, fg])
    root = ET.parse(tmp_path / "out" / "run.pvd").getroot()
    ds = root.findall("Collection/DataSet")
    assert [(d.get("timestep"), d.get("file")) for d in ds] == [("0.0", "run_0.vtm"), ("0.5", "run_1.vtm")]
    mb = ET.parse(tmp_path / "out" / "run_1.vtm").getroot().findall("vtkMultiBlockDataSet/DataSet")
    assert [d.get("file") for d in mb] == ["particles_1.vtu", "grid_1.vts"]


def test_write_ply(tb, tmp_path):
    from tesserae_b200 import export
    x = np.array([[0.0, 1.5], [2.0, -1.0]])  # 2D, two points
    path = export.write_ply(str(tmp_path / "pts"), x)
    raw = path.read_bytes()
    header = (b"ply\nformat binary_little_endian 1.0\nelement vertex 2\n"
              b"property float x\nproperty float y\nproperty float z\nend_header\n")
    assert raw.startswith(header)
    body = np.frombuffer(raw[len(header):], dtype="<f4")
    assert np.array_equal(body, [0.0, 2.0, 0.0, 1.5, -1.0, 0.0])
