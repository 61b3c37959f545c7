"""The CPU oracle against the reference's own known answers (tests/golden/
known_answers.json, extracted from Tesserae.jl's test files and doctests)."""
import json
import pathlib

import numpy as np
import pytest

from helpers import basis_kind

CASES = json.loads((pathlib.Path(__file__).parent / "golden" / "known_answers.json").read_text())["cases"]


def by_kind(kind):
    return [c for c in CASES if c["kind"] == kind]


def mesh2(tb, h, lims, L=2):
    lims = [tuple(l) for l in lims]
    if len(lims) == 1:  # 1-D cases run on a 2-D mesh with an interior second coordinate
        lims = lims + [lims[0]]
    return tb.CartesianMesh(h, *lims, block_size_log2=L)


def test_jets(oracle):
    for c in by_kind("jet_bspline_quadratic"):
        assert oracle.jet_bspline_quadratic(c["xi"]) == (c["value"], c["deriv"]), c["source"]
    for c in by_kind("jet_ugimp"):
        assert oracle.jet_ugimp(c["xi"], c["l"]) == (c["value"], c["deriv"]), c["source"]


def test_ugimp_support_sizes(tb, oracle):
    for c in by_kind("ugimp_support_size"):
        mesh = mesh2(tb, c["h"], [c["lims"], c["lims"]])
        win = oracle.supportnodes(mesh, tb._abi.TB_UGIMP, [c["x"], 0.55], c["l"])
        assert win[0][1] - win[0][0] + 1 == c["size"], c["source"]


def test_mesh_doctests(tb, oracle):
    for c in by_kind("mesh_size"):
        assert list(mesh2(tb, c["h"], c["lims"]).n_nodes) == c["size"], c["source"]
    for c in by_kind("supportnodes_radius"):
        # supportnodes(x, r, mesh) is the uGIMP window with r = 1 + l/2 (l in units of h).
        mesh = mesh2(tb, c["h"], c["lims"])
        lnorm = 2.0 * (c["r"] - 1)
        win = oracle.supportnodes(mesh, tb._abi.TB_UGIMP, [c["x"][0], 2.5], lnorm * c["h"])
        assert [list(win[0])] == c["range"], c["source"]
    for c in by_kind("findcell") + by_kind("findblock"):
        L = c.get("block_size_log2", 0)  # block_size_log2 = 0 makes blocks equal cells
        mesh = mesh2(tb, c["h"], c["lims"], L=L)
        P = tb.Particles(1, 2)
        P.x[:, 0] = c["x"]
        part = tb.Partition(mesh, 1)
        oracle.bin(mesh, P, part)
        b = int(part.blockids[0]) - 1
        nb = mesh.nblocks()
        got = [b % nb[0] + 1, b // nb[0] + 1]
        assert got == c.get("cell", c.get("block")), c["source"]


def _props(tb, oracle, c):
    dim, h = c["dim"], c["h"]
    mesh = tb.CartesianMesh(h, *[(0.0, 1.0)] * dim)
    P = tb.Particles(1, dim)
    P.x[:, 0] = c["x"]
    prm = tb.step_params(1.0, gimp_l=c["l"], basis=basis_kind(tb._abi, c["basis"]))
    W = tb.generate_basis_weights(dim, 1)
    oracle.update_weights(mesh, P, prm, W)
    return mesh, W


def check_props(tb, mesh, W, x, c):
    dim = mesh.dim
    win = W.window[0].reshape(dim, 2)
    w = W.w[0]
    gw = W.grad_w[0]
    eps = np.finfo(np.float64).eps
    pu = np.isclose(w.sum(), 1.0, rtol=np.sqrt(eps), atol=0) and np.all(
        np.isclose(gw.sum(axis=0) + 1.0, 1.0, rtol=np.sqrt(eps), atol=0))
    Xw = np.zeros(dim)
    XgW = np.zeros((dim, dim))
    for s in range(3 ** dim):
        loc = [(s // 3 ** d) % 3 for d in range(dim)]
        if any(loc[d] > win[d][1] - win[d][0] for d in range(dim)):
            continue
        X = np.array([mesh.xmin[d] + (win[d][0] - 1 + loc[d]) * mesh.h for d in range(dim)])
        Xw += X * w[s]
        XgW += np.outer(X, gw[s])
    lfr = np.allclose(Xw, x, rtol=np.sqrt(eps), atol=0) and np.allclose(XgW, np.eye(dim), rtol=np.sqrt(eps),
                                                                         atol=np.sqrt(eps))
    truncated = any(win[d][1] - win[d][0] + 1 != 3 for d in range(dim))
    return pu, lfr, truncated


@pytest.mark.parametrize("case", by_kind("basis_props"), ids=lambda c: f"{c['basis']}-{c['dim']}d-{c['source']}")
def test_basis_properties(tb, oracle, case):
    mesh, W = _props(tb, oracle, case)
    pu, lfr, truncated = check_props(tb, mesh, W, np.array(case["x"]), case)
    assert pu == case["pu"], case["source"]
    assert lfr == case["lfr"], case["source"]
    if case["truncated"] is not None:
        assert truncated == case["truncated"], case["source"]


@pytest.mark.parametrize("case", by_kind("kc_positive"),
                         ids=lambda c: f"{c['dim']}d-{len(c['nodes'])}nodes-{c['source']}")
def test_kernel_correction_positive(tb, oracle, case):
    """The node weight of KernelCorrection(BSpline(Quadratic())) is > -sqrt(eps)
    for every particle of the 1/11 lattice around the node, as in the
    reference's positivity test."""
    dim, L = case["dim"], case["L"]
    mesh = tb.CartesianMesh(case["h"], *[tuple(l) for l in case["lims"]])
    eps = np.finfo(np.float64).eps
    prm = tb.step_params(1.0, basis=tb._abi.TB_KC_BSPLINE_QUADRATIC)
    for node in case["nodes"]:
        axes = []
        for d in range(dim):
            lo = max(case["lims"][d][0], node[d] - L - 1)
            hi = min(case["lims"][d][1], node[d] + L - 1) - np.sqrt(eps)
            axes.append(np.arange(0, int(np.floor((hi - lo) * 11 + 1e-9)) + 1) / 11.0 + lo)
        pts = np.stack([g.ravel() for g in np.meshgrid(*axes, indexing="ij")])
        n = pts.shape[1]
        P = tb.Particles(n, dim)
        P.x[...] = pts
        W = tb.generate_basis_weights(dim, n)
        oracle.update_weights(mesh, P, prm, W)
        win = W.window.reshape(n, dim, 2)
        val = np.zeros(n)
        for i in range(n):
            loc = [node[d] - win[i, d, 0] for d in range(dim)]  # 0-based slot of the node in the window
            if all(0 <= loc[d] <= win[i, d, 1] - win[i, d, 0] for d in range(dim)):
                val[i] = W.w[i][sum(loc[d] * 3 ** d for d in range(dim))]
        assert np.all(val > -np.sqrt(eps)), (node, case["source"], val.min())


def test_tile_contains_every_window(tb, oracle):
    c = by_kind("tile_contains")[0]
    mesh = tb.CartesianMesh(c["h"], *[tuple(l) for l in c["lims"]], block_size_log2=2)
    ax = tb.scenes.grid_sampling_axis(0.0, 1.0, c["h"])
    pts = tb.scenes._lattice([ax, ax])
    n = pts.shape[1]
    P = tb.Particles(n, 2)
    P.x[...] = pts
    part = tb.Partition(mesh, n)
    oracle.bin(mesh, P, part)
    for name in c["bases"]:
        prm = tb.step_params(1.0, gimp_l=c["l"], basis=basis_kind(tb._abi, name))
        W = tb.generate_basis_weights(2, n)
        oracle.update_weights(mesh, P, prm, W)
        nb = mesh.nblocks()
        b = part.blockids.astype(np.int64) - 1
        ok = part.blockids > 0
        for d, bd in enumerate([b % nb[0], b // nb[0]]):
            lo = bd * 4 - 1 + 1  # 1-based first tile node of the block: 4 B - 1 (0-based)
            hi = lo + 4 + 2
            start, stop = W.window[:, 2 * d], W.window[:, 2 * d + 1]
            assert np.all((start[ok] >= lo[ok]) & (stop[ok] <= hi[ok])), (name, c["source"])


def test_partition_lists_ascending(tb, oracle):
    from helpers import reference_partition
    c = by_kind("partition_lists")[0]
    rng = np.random.default_rng(1234)
    mesh = tb.CartesianMesh(0.1, (0.0, 2.0), (0.0, 3.0))
    n = 3000
    P = tb.Particles(n, 2)
    P.x[...] = rng.uniform(-0.2, 3.2, size=(2, n))  # some outside the mesh
    part = tb.Partition(mesh, n)
    na, nass = oracle.bin(mesh, P, part)
    bid, counts, offsets, blocklist, perm = reference_partition(mesh, P.x)
    assert np.array_equal(part.blockids, bid), c["source"]
    assert np.array_equal(part.counts, counts)
    assert np.array_equal(part.offsets, offsets)
    assert na == len(blocklist) and np.array_equal(part.blocklist[:na], blocklist)
    assert nass == len(perm) and np.array_equal(part.particleindices[:nass], perm)


def test_block_ordered_scene_is_the_partition_order(tb, oracle):
    """scenes.block_ordered stores the particles in the order reorder_particles!
    leaves them in (gpu_block_strategy.jl:204-238): after it, the oracle's
    partition lists the particles 1..n in order, and the particle set (positions
    with their velocities) is unchanged."""
    sc = tb.scenes.cube3d(scale=16)
    before = {tuple(np.r_[sc.particles.x[:, p], sc.particles.v[:, p]]) for p in range(sc.particles.n)}
    part0 = tb.Partition(sc.mesh, sc.particles.n)
    oracle.bin(sc.mesh, sc.particles, part0)
    assert not np.array_equal(part0.particleindices, np.arange(1, sc.particles.n + 1))
    tb.scenes.block_ordered(sc)
    part = tb.Partition(sc.mesh, sc.particles.n)
    oracle.bin(sc.mesh, sc.particles, part)
    assert np.array_equal(part.particleindices, np.arange(1, sc.particles.n + 1))
    after = {tuple(np.r_[sc.particles.x[:, p], sc.particles.v[:, p]]) for p in range(sc.particles.n)}
    assert before == after


def test_block_order_is_the_same_workload(tb, oracle):
    """The bench stores the particles in block order: the same particles advance
    the same way (2 FP64 oracle steps), up to the order of the P2G sums."""
    a = tb.scenes.cube3d(scale=16)
    b = tb.scenes.block_ordered(tb.scenes.cube3d(scale=16))
    order = tb.scenes._sort_by_block(a.mesh, a.particles.x)
    assert np.array_equal(b.particles.x, a.particles.x[:, order])
    for sc in (a, b):
        G = tb.generate_grid(sc.mesh)
        oracle.step_parallel(sc.mesh, sc.particles, G, sc.params, 2, 1)
    for k in ("x", "v", "F"):
        ref = getattr(a.particles, k)[..., order]
        got = getattr(b.particles, k)
        assert np.allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max()), k


def test_grid_sampling_doctest(tb):
    """generate_particles(ParticleProp, mesh; alg=GridSampling()) doctest
    (src/particles.jl:79-89): 96 particles, the first at (0.125, 0.125)."""
    for c in by_kind("grid_sampling"):
        mesh = tb.CartesianMesh(c["h"], *[tuple(l) for l in c["lims"]])
        P = tb.generate_particles(mesh, tb.GridSampling(c["spacing"]))
        assert P.n == c["n"], c["source"]
        assert list(P.x[:, 0]) == c["first"], c["source"]
        assert np.all(P.v == 0) and np.all(P.F[[0, 3]] == 1) and np.all(P.F[[1, 2]] == 0)
