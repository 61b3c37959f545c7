"""reorder_particles! and block_ordered_particle_contiguity on the device
(src/Parallel/gpu_block_strategy.jl:172-238), checked the way the reference's
test/partition.jl:4-30 checks its CPU form: every field must travel with its
particle; the score follows the reference's GPU estimator; the fused step with
the reorder policy gives the same particles as the step without it."""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def shuffled_cube(tb, dtype=np.float64, x64=False, seed=3):
    sc = tb.scenes.cube3d(scale=8)
    P = sc.particles
    n = P.n
    rng = np.random.default_rng(seed)
    order = rng.permutation(n)
    P.x[...] = P.x[:, order]
    P.v[...] = 10.0 * P.x          # v = 10 x, as the reference's test sets it
    P.V[...] = -np.arange(n, dtype=np.float64) - 1.0
    P.sigma[...] = rng.normal(size=P.sigma.shape)
    P.F[...] = P.F + rng.normal(scale=1e-3, size=P.F.shape)
    return sc, P.to("torch", device="cuda", dtype=dtype, x64=x64)


def same_block_fraction(blockids, counts):
    """The reference's GPU score: neighbours in memory sharing a (non-zero)
    block over nassigned - nactive (gpu_block_strategy.jl:178-191)."""
    b = np.asarray(blockids)
    same = int(np.sum((b[:-1] != 0) & (b[:-1] == b[1:])))
    nassigned = int(np.sum(b != 0))
    nactive = int(np.sum(np.asarray(counts) > 0))
    maxsame = nassigned - nactive
    return 1.0 if maxsame <= 0 else same / maxsame


@pytest.mark.parametrize("dtype,x64", [(np.float64, False), (np.float32, False), (np.float32, True)])
def test_reorder_fields_travel_together(tb, ctx, dtype, x64):
    from tesserae_b200 import runtime
    sc, P = shuffled_cube(tb, dtype, x64)
    n = P.n
    before = {k: getattr(P, k).double().cpu().numpy().copy() for k in ("x", "v", "V", "sigma", "F")}
    part = tb.Partition(sc.mesh, n, backend="torch", device="cuda")
    runtime.update(part, P, sc.mesh, ctx=ctx)
    perm = part.particleindices.cpu().numpy() - 1
    assert runtime.reorder_particles(P, part, 1.0, ctx=ctx)
    after = {k: getattr(P, k).double().cpu().numpy() for k in before}
    for k in before:
        assert np.array_equal(after[k], before[k][..., perm]), k  # exact: a permutation
    d = part.numpy()
    assert np.array_equal(d["particleindices"], np.arange(1, n + 1))
    assert np.all(np.diff(d["blockids"]) >= 0)  # block order in memory
    np.testing.assert_array_equal(after["v"], after["x"] * 10.0)  # float: v was set to 10 x before the cast
    # the partition still describes the particles: re-binning reproduces it
    part2 = tb.Partition(sc.mesh, n, backend="torch", device="cuda")
    runtime.update(part2, P, sc.mesh, ctx=ctx)
    d2 = part2.numpy()
    for k in ("blockids", "counts", "offsets", "particleindices"):
        assert np.array_equal(d2[k], d[k]), k


def test_contiguity_score_and_policy(tb, ctx):
    from tesserae_b200 import runtime
    sc, P = shuffled_cube(tb)
    n = P.n
    part = tb.Partition(sc.mesh, n, backend="torch", device="cuda")
    runtime.update(part, P, sc.mesh, ctx=ctx)
    d = part.numpy()
    want = same_block_fraction(d["blockids"], d["counts"])
    got = runtime.block_ordered_particle_contiguity(part, n, ctx=ctx)
    assert got == pytest.approx(want, rel=1e-12) and got < 0.2
    assert not runtime.reorder_particles(P, part, 0.0, ctx=ctx)      # threshold 0 never reorders
    assert runtime.reorder_particles(P, part, 0.85, ctx=ctx)         # score below the threshold
    assert runtime.block_ordered_particle_contiguity(part, n, ctx=ctx) == 1.0
    assert not runtime.reorder_particles(P, part, 0.85, ctx=ctx)     # already block-ordered
    assert runtime.reorder_particles(P, part, 1.0, ctx=ctx)          # threshold 1 always does


def test_reorder_refuses_particles_outside(tb, ctx):
    from tesserae_b200 import runtime
    sc, P = shuffled_cube(tb)
    P.x[0, 5] = -1.0  # outside the mesh: block 0
    part = tb.Partition(sc.mesh, P.n, backend="torch", device="cuda")
    runtime.update(part, P, sc.mesh, ctx=ctx)
    with pytest.raises(RuntimeError, match="outside the mesh"):
        runtime.reorder_particles(P, part, 1.0, ctx=ctx)
    assert not runtime.reorder_particles(P, part, 0.0, ctx=ctx)  # nothing due: no error


@pytest.mark.parametrize("dtype,x64,tol", [(np.float64, False, 1e-11), (np.float32, True, 1e-5)])
def test_step_with_reorder_policy_matches_plain_step(tb, ctx, dtype, x64, tol):
    """Shuffled particles stepped with the 0.85 policy (reordered at the first
    binning) against the same particles stepped without it; particles are
    matched through an id carried in the uGIMP length field `l`, which the
    B-spline step does not read."""
    from tesserae_b200 import runtime
    sc = tb.scenes.cube3d(scale=8)
    Pn = sc.particles
    n = Pn.n
    order = np.random.default_rng(4).permutation(n)
    Pn.x[...] = Pn.x[:, order]
    Pn.v[...] = Pn.v[:, order]
    Pq = tb.Particles(n, 3, optional=("l",))
    for k in ("x", "v", "V", "sigma", "F"):
        getattr(Pq, k)[...] = getattr(Pn, k)
    Pq.l[...] = np.arange(n, dtype=np.float64)
    res = []
    for thr in (None, 0.85):
        P = Pq.to("torch", device="cuda", dtype=dtype, x64=x64)
        part = tb.Partition(sc.mesh, n, backend="torch", device="cuda")
        G = tb.generate_grid(sc.mesh, dtype, backend="torch", device="cuda")
        runtime.step(G, P, part, sc.mesh, sc.params, 5, ctx=ctx, reorder_threshold=thr)
        ctx.synchronize()
        ids = P.l.cpu().numpy().astype(np.int64)
        inv = np.empty(n, dtype=np.int64)
        inv[ids] = np.arange(n)
        res.append({k: getattr(P, k).double().cpu().numpy()[..., inv] for k in ("x", "v", "F")})
        if thr is not None:
            assert runtime.block_ordered_particle_contiguity(part, n, ctx=ctx) > 0.85
    for k in ("x", "v", "F"):
        assert rel_l2(res[1][k], res[0][k]) <= tol, k
