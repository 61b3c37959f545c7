"""Block-sparse grid numbering (no GPU): the oracle restatement of
update_sparsity! (oracle/spgrid.py) against the reference test's own
construction of the expected active set (test/sparray.jl:70-107), the stored
node count, numbering reuse for an unchanged active set, and the host mirror's
sparse grid layout."""
import pathlib
import sys

import numpy as np

sys.path.insert(0, str(pathlib.Path(__file__).resolve().parent.parent / "oracle"))
import spgrid  # noqa: E402


def circle_particles(tb):
    """generate_particles(CartesianMesh(0.25, (0,4), (0,4))) filtered to the
    disk (x-2)^2 + (y-2)^2 < 1 (test/sparray.jl:71-75)."""
    mesh = tb.CartesianMesh(0.25, (0.0, 4.0), (0.0, 4.0))
    x = tb.generate_points(tb.GridSampling(), mesh)
    keep = (x[0] - 2) ** 2 + (x[1] - 2) ** 2 < 1
    return mesh, x[:, keep]


def expected_active_as_in_reference_test(mesh, x):
    """The test's loop: every particle's findblock I marks (I - 1):(I + 1)
    clipped to the block range, once per newly occupied block."""
    nb = mesh.nblocks()
    occupied = np.zeros(nb, dtype=bool)
    active = np.zeros(nb, dtype=bool)
    L = mesh.block_size_log2
    for p in range(x.shape[1]):
        c = [int(np.floor((x[d, p] - mesh.xmin[d]) * mesh.h_inv)) for d in range(mesh.dim)]
        if any(ci < 0 or ci > mesh.n_nodes[d] - 2 for d, ci in enumerate(c)):
            continue
        I = tuple(ci >> L for ci in c)
        if not occupied[I]:
            occupied[I] = True
            sl = tuple(slice(max(i - 1, 0), min(i + 2, nb[d])) for d, i in enumerate(I))
            active[sl] = True
    return occupied.ravel(order="F"), active.ravel(order="F")


def test_circle_active_set_matches_reference_test(tb):
    mesh, x = circle_particles(tb)
    occ_ref, act_ref = expected_active_as_in_reference_test(mesh, x)
    occ = spgrid.occupied_blocks(mesh, x)
    num, blist, k = spgrid.numbering(mesh, x)
    assert np.array_equal(occ, occ_ref)
    assert np.array_equal(num != 0, act_ref)
    bl = 1 << (mesh.block_size_log2 * mesh.dim)
    assert k * bl == act_ref.sum() * bl  # n_particles == count(expected_active) * blocklength
    assert np.array_equal(num[blist - 1], np.arange(1, k + 1))  # storage order = ascending block id


def test_numbering_unchanged_when_active_set_unchanged(tb):
    """test/sparray.jl:109-131: (1,1), (2,1), (9,1) on CartesianMesh(1, (0,16), (0,4));
    moving the first particle to (10,1) keeps the occupied set, so the numbering."""
    mesh = tb.CartesianMesh(1.0, (0.0, 16.0), (0.0, 4.0))
    x1 = np.array([[1.0, 2.0, 9.0], [1.0, 1.0, 1.0]])
    x2 = np.array([[10.0, 2.0, 9.0], [1.0, 1.0, 1.0]])
    n1, _, k1 = spgrid.numbering(mesh, x1)
    n2, _, k2 = spgrid.numbering(mesh, x2)
    assert k1 == k2 and np.array_equal(n1, n2)
    assert spgrid.numbering(mesh, np.zeros((2, 0)))[2] == 0  # no particles: nothing stored


def test_storage_index_layout(tb):
    """(k - 1) blocklength + column-major local index (src/Grids/spindices.jl:87-100),
    and the host mirror's dense() view places every stored node back."""
    mesh = tb.CartesianMesh(1.0, (0.0, 16.0), (0.0, 8.0))
    x = np.array([[5.5, 13.5], [2.5, 6.5]])
    num, blist, k = spgrid.numbering(mesh, x)
    W = 1 << mesh.block_size_log2
    g = tb.generate_grid(mesh, np.float64, sparse=True, capacity=k * W * W)
    g.block_numbering[:] = num
    g.active_blocks[:k] = blist
    g.nactive[0] = k
    rng = np.random.default_rng(1)
    g.m[:] = rng.normal(size=g.m.shape)
    dense = g.dense()["m"]
    for node in [(4, 2), (7, 3), (12, 7), (16, 8), (0, 0)]:
        s = spgrid.storage_index(mesh, num, node)
        lin = node[0] + mesh.n_nodes[0] * node[1]
        assert dense[lin] == (0.0 if s < 0 else g.m[s])
