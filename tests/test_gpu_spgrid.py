"""Block-sparse grid (SpGrid) on the device, through the C ABI.

tb_update_sparsity_* against the numpy restatement of update_sparsity!
(oracle/spgrid.py): numbering, active list and count bit for bit. Steps on a
sparse grid against the same steps on a dense grid from the same state: FP64
particle fields to 1e-12 relative L2 (only the order of the atomic sums
differs), the mixed forms to 1e-6, and the last step's grid on every node
(stored nodes to the same bounds, unstored nodes zero on both). A scatter into a
node whose block the grid does not store, and a grid too small for its active
blocks, are reported as errors (the kernels skip those nodes)."""
import pathlib
import sys

import numpy as np
import pytest

from helpers import rel_l2

sys.path.insert(0, str(pathlib.Path(__file__).resolve().parent.parent / "oracle"))
import spgrid  # noqa: E402

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SCENES = {"clusters3d": 8, "readme2d": 2, "cube3d": 8, "dambreak3d": 8}


def scene(tb, name):
    return getattr(tb.scenes, name)(scale=SCENES[name])


@pytest.mark.parametrize("form", ["f64", "f32", "x64"])
@pytest.mark.parametrize("name", ["clusters3d", "readme2d"])
def test_update_sparsity_matches_oracle(tb, ctx, name, form):
    from tesserae_b200 import runtime
    sc = scene(tb, name)
    if form == "x64" and sc.mesh.dim != 3:
        pytest.skip("3D scene")
    dtype = np.float64 if form == "f64" else np.float32
    P = sc.particles.to("torch", device="cuda", dtype=dtype, x64=form == "x64")
    part = tb.Partition(sc.mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(sc.mesh, dtype, backend="torch", device="cuda", sparse=True)
    nstored = runtime.update_sparsity(G, P, part, sc.mesh, ctx=ctx)
    xh = P.x.cpu().numpy()
    num, blist, k = spgrid.numbering(sc.mesh, xh)
    g = G.numpy()
    assert int(g["nactive"][0]) == k
    assert nstored == k * G.blocklength
    assert np.array_equal(g["block_numbering"], num)
    assert np.array_equal(g["active_blocks"][:k], blist)
    assert G.capacity >= nstored
    if name == "clusters3d":  # a sparse scene stores a fraction of the dense grid
        assert nstored < 0.5 * sc.mesh.nnodes


def run(tb, ctx, sc, form, sparse, nsteps):
    from tesserae_b200 import runtime
    dtype = np.float64 if form == "f64" else np.float32
    P = sc.particles.to("torch", device="cuda", dtype=dtype, x64=form == "x64")
    part = tb.Partition(sc.mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(sc.mesh, dtype, backend="torch", device="cuda", sparse=sparse)
    runtime.step(G, P, part, sc.mesh, sc.params, nsteps, ctx=ctx)
    ctx.synchronize()
    return P.to("numpy"), G.dense()


@pytest.mark.parametrize("name,form", [("clusters3d", "f64"), ("clusters3d", "x64"), ("readme2d", "f64"),
                                       ("cube3d", "f32"), ("dambreak3d", "f64"), ("dambreak3d", "x64")])
def test_sparse_steps_match_dense(tb, ctx, name, form):
    sc = scene(tb, name)
    tol = 1e-12 if form == "f64" else 1e-6
    nsteps = 4
    Pd, Gd = run(tb, ctx, sc, form, False, nsteps)
    Ps, Gs = run(tb, ctx, sc, form, True, nsteps)
    for k in ("x", "v", "F"):
        assert rel_l2(getattr(Ps, k), getattr(Pd, k)) <= tol, (name, form, k)
    for k in ("m", "mv", "f", "v", "vn"):
        assert rel_l2(Gs[k], Gd[k]) <= (1e-12 if form == "f64" else 1e-5), (name, form, k)
    # nodes the sparse grid leaves out carry nothing on the dense grid either
    assert np.count_nonzero(Gs["m"]) == np.count_nonzero(Gd["m"])


def test_stale_sparsity_is_reported(tb, ctx):
    """A P2G whose particles moved to blocks the grid does not store: the
    scatter skips those nodes and the status word reports it."""
    from tesserae_b200 import runtime
    sc = scene(tb, "cube3d")  # the cube [1/4, 3/4]^3 of the domain
    P = sc.particles.to("torch", device="cuda", dtype=np.float64)
    part = tb.Partition(sc.mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(sc.mesh, np.float64, backend="torch", device="cuda", sparse=True)
    runtime.update_sparsity(G, P, part, sc.mesh, ctx=ctx)
    # move the cube by a fifth of the domain in -x: its left part lies in blocks
    # the grid does not store
    (a, b) = sc.mesh.lims[0]
    P.x[0].sub_(0.2 * (b - a))
    runtime.update(part, P, sc.mesh, ctx=ctx)
    with pytest.raises(RuntimeError, match="inactive sparse-grid block"):
        runtime.P2G(G, P, part, sc.mesh, sc.params, grid_half=False, ctx=ctx)
        ctx.synchronize()
    ctx.synchronize()  # the status word was cleared by the report


def test_capacity_is_checked(tb, ctx):
    """tb_update_sparsity_* refuses a grid too small for its active blocks
    (TB_ERR_CAPACITY) after writing the numbering and the needed count."""
    import ctypes as C
    from tesserae_b200 import _abi
    sc = scene(tb, "clusters3d")
    P = sc.particles.to("torch", device="cuda", dtype=np.float64)
    part = tb.Partition(sc.mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(sc.mesh, np.float64, backend="torch", device="cuda", sparse=True)
    assert G.capacity == G.blocklength
    n = C.c_int64(0)
    rc = ctx.lib.tb_update_sparsity_f64(ctx.ptr, C.byref(sc.mesh.struct()), C.byref(P.struct()),
                                        C.byref(part.struct()), C.byref(G.struct()), C.byref(n))
    assert rc == _abi.TB_ERR_CAPACITY
    num, _, k = spgrid.numbering(sc.mesh, P.x.cpu().numpy())
    assert n.value == k * G.blocklength
    assert np.array_equal(G.numpy()["block_numbering"], num)


def test_reverse_step_refuses_sparse_grid(tb, ctx):
    from tesserae_b200 import runtime
    sc = scene(tb, "cube3d")
    P = sc.particles.to("torch", device="cuda", dtype=np.float64)
    part = tb.Partition(sc.mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(sc.mesh, np.float64, backend="torch", device="cuda", sparse=True)
    runtime.update_sparsity(G, P, part, sc.mesh, ctx=ctx)
    adj = tb.Adjoint(P.n, 3, backend="torch", device="cuda")
    with pytest.raises(RuntimeError, match="dense grid"):
        runtime.adjoint_step(G, P, part, sc.mesh, sc.params, adj, ctx=ctx)
