"""Full-size checks of the headline configuration (cube3d: 256^3 cells,
16 777 216 particles) and the atomic-contention configuration (clusters3d:
512^3 cells, 33.5 M particles):

* the plain FP64 device step against the FP64 oracle's OpenMP step for 3 steps
  from the same block-ordered state (relative L2 <= 1e-9 in x, v, F);
* size-independent conservation laws of the FP32 P2G at full size: the grid
  mass equals the particle mass, the grid momentum the particle momentum, and
  the grid force the total gravity force (the B-spline weights sum to one and
  their gradients to zero on interior windows), each to 1e-5 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def cube(tb):
    return tb.scenes.block_ordered(tb.scenes.cube3d())


def test_fp64_step_matches_oracle_full_size(tb, ctx, oracle, cube):
    from tesserae_b200 import runtime
    import conftest
    mesh, prm = cube.mesh, cube.params
    P = cube.particles.to("torch", device="cuda", dtype=np.float64)
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(mesh, np.float64, backend="torch", device="cuda")
    runtime.step(G, P, part, mesh, prm, 3, ctx=ctx)
    ctx.synchronize()
    got = P.numpy()
    del P, part, G
    torch.cuda.empty_cache()
    Pc = cube.particles.to("numpy")
    Gc = tb.generate_grid(mesh)
    oracle.step_parallel(mesh, Pc, Gc, prm, 3, conftest.load_oracle_module().cores())
    for k in ("x", "v", "F"):
        ref = getattr(Pc, k)
        err = np.linalg.norm(got[k] - ref) / np.linalg.norm(ref)
        assert err <= 1e-9, (k, err)


def _p2g_sums(tb, runtime, ctx, sc, x64):
    mesh, prm = sc.mesh, sc.params
    P = sc.particles.to("torch", device="cuda", dtype=np.float32, x64=x64)
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(mesh, np.float32, backend="torch", device="cuda")
    if x64:
        # the FP64-position form runs through the fused step only: one step's
        # P2G leaves m, mv, f of the step's start in the grid
        Q = sc.particles.to("torch", device="cuda", dtype=np.float32, x64=True)
        runtime.step(G, Q, part, mesh, prm, 1, ctx=ctx)
    else:
        runtime.update(part, P, mesh, ctx=ctx)
        runtime.P2G(G, P, part, mesh, prm, grid_half=False, ctx=ctx)
    ctx.synchronize()
    m = G.m.double().sum().item()
    mv = G.mv.double().sum(dim=1).cpu().numpy()
    f = G.f.double().sum(dim=1).cpu().numpy()
    mp = (P.m.double() if P.m is not None else torch.full((P.n,), prm.mass, dtype=torch.float64,
                                                           device="cuda"))
    pv = (mp[None, :] * P.v.double()).sum(dim=1).cpu().numpy()
    pscale = (mp[None, :] * P.v.double().abs()).sum(dim=1).cpu().numpy()
    return m, mv, f, mp.sum().item(), pv, pscale, np.array(prm.gravity[:3])


@pytest.mark.parametrize("scene,x64", [("cube3d", True), ("cube3d", False), ("clusters3d", False)])
def test_p2g_conservation_full_size(tb, ctx, cube, scene, x64):
    from tesserae_b200 import runtime
    sc = cube if scene == "cube3d" else tb.scenes.clusters3d()
    m, mv, f, mtot, ptot, pscale, g = _p2g_sums(tb, runtime, ctx, sc, x64)
    assert abs(m - mtot) <= 1e-5 * mtot
    # random velocities cancel in the sum: the tolerance is relative to sum m |v|
    assert np.all(np.abs(mv - ptot) <= 1e-5 * pscale)
    fg = mtot * g
    assert np.linalg.norm(f - fg) <= 1e-5 * np.linalg.norm(fg)
    torch.cuda.empty_cache()
