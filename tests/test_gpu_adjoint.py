"""Reverse mode on the device (through the C ABI) against the oracle and
against finite differences.

Tolerances, per test: one adjoint step against the oracle's adjoint step on
the same state, relative L2 per field <= 1e-10 in FP64 (only the order of the
atomic sums differs) and <= 1e-4 in the mixed FP32 form (the forward grid is
rebuilt in FP32 on both sides, with different atomic orders, and the grid
sensitivities divide by nodal masses); the checkpointed tape against the
oracle's stored-state rollout gradient <= 1e-9 (FP64); tapes with different
checkpoint intervals agree to 1e-12; directional derivatives against central
finite differences of the FP64 device rollout within 1e-6 relative (FP64
tape) and 1e-4 (FP32 tape).
"""
import numpy as np
import pytest

from adjoint_helpers import box_scene, linear_loss, make_consistent, oracle_rollout_grad, random_seeds
from helpers import rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

CASES = {
    "bspline3d": dict(dim=3),
    "pic_blend": dict(dim=3, alpha=0.9),
    "ugimp": dict(dim=3, basis=1),
    "fluid": dict(dim=3, material=1),
    "walls": dict(dim=3, lo=0.02, hi=0.4, walls=0b111111),
    "bspline2d": dict(dim=2, cells=16),
    # 4^3 particles per cell in lattice order: 4096 per block, so the scatter
    # takes each block in several passes
    "dense": dict(dim=3, ppc=4),
}


def device_adjoint(tb, P, seeds):
    adj = tb.Adjoint(P.n, P.dim, backend="torch", device="cuda")
    adj.x.copy_(torch.from_numpy(seeds["x"]))
    adj.v.copy_(torch.from_numpy(seeds["v"]))
    adj.F.copy_(torch.from_numpy(seeds["F"]))
    return adj


def host_adjoint(tb, P, seeds):
    adj = tb.Adjoint(P.n, P.dim)
    adj.x[...] = seeds["x"]
    adj.v[...] = seeds["v"]
    adj.F[...] = seeds["F"]
    return adj


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-10), (np.float32, 1e-4)])
def test_adjoint_step_matches_oracle(tb, oracle, ctx, case, dtype, tol):
    from tesserae_b200 import runtime
    mesh, P, prm = box_scene(tb, dtype=dtype, **CASES[case])
    seeds = random_seeds(P, np.random.default_rng(3))
    adj_o = host_adjoint(tb, P, seeds)
    oracle.adjoint_step(mesh, P, tb.generate_grid(mesh, dtype), prm, adj_o)
    Pd = P.to("torch", device="cuda")
    adj_d = device_adjoint(tb, P, seeds)
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(mesh, dtype, backend="torch", device="cuda")
    runtime.adjoint_step(G, Pd, part, mesh, prm, adj_d, ctx=ctx)
    ctx.synchronize()
    got = adj_d.numpy()
    for k in ("x", "v", "F", "mu", "lam"):
        assert rel_l2(got[k], getattr(adj_o, k)) <= tol, (case, k, rel_l2(got[k], getattr(adj_o, k)))


def test_adjoint_step_accumulates_lame(tb, ctx):
    """mu / lambda sensitivities add to what the arrays held."""
    from tesserae_b200 import runtime
    mesh, P, prm = box_scene(tb)
    seeds = random_seeds(P, np.random.default_rng(4))
    out = []
    for pre in (0.0, 1.0):
        adj = device_adjoint(tb, P, seeds)
        adj.mu.fill_(pre)
        adj.lam.fill_(pre)
        runtime.adjoint_step(tb.generate_grid(mesh, np.float64, backend="torch", device="cuda"),
                             P.to("torch", device="cuda"), tb.Partition(mesh, P.n, backend="torch", device="cuda"),
                             mesh, prm, adj, ctx=ctx)
        ctx.synchronize()
        out.append(adj.numpy())
    assert np.allclose(out[1]["mu"], out[0]["mu"] + 1.0, rtol=0, atol=1e-9 * np.abs(out[0]["mu"]).max())
    assert np.allclose(out[1]["lam"], out[0]["lam"] + 1.0, rtol=0, atol=1e-9 * np.abs(out[0]["lam"]).max())


def tape_grad(tb, ctx, mesh, P, prm, nsteps, every, seeds):
    from tesserae_b200 import runtime
    Pd = P.to("torch", device="cuda")
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(mesh, P.dtype, backend="torch", device="cuda")
    runtime.tape_forward(G, Pd, part, mesh, prm, nsteps, every, ctx=ctx)
    final = Pd.to("numpy")
    adj = device_adjoint(tb, P, seeds)
    runtime.tape_backward(G, Pd, part, mesh, prm, adj, ctx=ctx)
    ctx.synchronize()
    restored = Pd.to("numpy")
    return adj.numpy(), final, restored


@pytest.mark.parametrize("every", [3, 1])  # 1: the whole tape, no recompute in the backward pass
@pytest.mark.parametrize("case", ["bspline3d", "ugimp", "walls", "bspline2d"])
def test_tape_matches_oracle_rollout_grad(tb, oracle, ctx, case, every):
    mesh, P, prm = box_scene(tb, **CASES[case])
    nsteps = 7
    seeds = random_seeds(P, np.random.default_rng(5))
    got, final, restored = tape_grad(tb, ctx, mesh, P, prm, nsteps, every, seeds)
    ref, final_o = oracle_rollout_grad(tb, oracle, mesh, P, prm, nsteps, seeds)
    assert rel_l2(final.x, final_o.x) <= 1e-12
    assert np.array_equal(restored.x, P.x) and np.array_equal(restored.F, P.F)  # step-0 state is back
    for k in ("x", "v", "F", "mu", "lam"):
        assert rel_l2(got[k], getattr(ref, k)) <= 1e-9, (case, k, rel_l2(got[k], getattr(ref, k)))


def test_tape_independent_of_checkpoint_interval(tb, ctx):
    mesh, P, prm = box_scene(tb)
    seeds = random_seeds(P, np.random.default_rng(6))
    grads = [tape_grad(tb, ctx, mesh, P, prm, 6, every, seeds)[0] for every in (1, 4, 6)]
    for g in grads[1:]:
        for k in ("x", "v", "F", "mu", "lam"):
            assert rel_l2(g[k], grads[0][k]) <= 1e-12, k


def device_loss(tb, ctx, mesh, P, prm, nsteps, seeds):
    from tesserae_b200 import runtime
    Pd = P.to("torch", device="cuda")
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(mesh, P.dtype, backend="torch", device="cuda")
    runtime.step(G, Pd, part, mesh, prm, nsteps, ctx=ctx)
    ctx.synchronize()
    return linear_loss(Pd.to("numpy"), seeds)


def shifted(P, prm, field, delta, eps):
    Q = P.to("numpy", dtype=np.float64)
    arr = getattr(Q, field)
    arr[...] = arr + eps * delta
    make_consistent(Q, prm)
    return Q


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-6), (np.float32, 1e-4)])
def test_tape_gradient_matches_fp64_finite_differences(tb, ctx, dtype, tol):
    """Directional derivatives of a 12-step rollout loss: the tape (FP64 or mixed
    FP32) against central differences of the FP64 device rollout."""
    mesh, P64, prm = box_scene(tb, cells=16, dt=5e-4)
    nsteps, every = 12, 5
    rng = np.random.default_rng(7)
    seeds = random_seeds(P64, rng)
    got, _, _ = tape_grad(tb, ctx, mesh, P64.to("numpy", dtype=dtype), prm, nsteps, every, seeds)
    for field, eps in (("x", 1e-7), ("v", 1e-6), ("mu", 1e-5), ("lam", 1e-5)):
        delta = rng.normal(size=getattr(P64, field).shape)
        if field in ("mu", "lam"):
            delta = delta * getattr(P64, field)
        Lp = device_loss(tb, ctx, mesh, shifted(P64, prm, field, delta, eps), prm, nsteps, seeds)
        Lm = device_loss(tb, ctx, mesh, shifted(P64, prm, field, delta, -eps), prm, nsteps, seeds)
        fd = (Lp - Lm) / (2 * eps)
        ad = float(np.sum(got[field] * delta))
        assert abs(ad - fd) <= tol * max(abs(fd), 1e-3), (field, ad, fd)


def test_rollout_function_autograd(tb, ctx):
    """torch.autograd through the tape equals the tape called directly."""
    from tesserae_b200 import runtime
    mesh, P, prm = box_scene(tb)
    Pd = P.to("torch", device="cuda")
    v0 = Pd.v.detach().clone().requires_grad_(True)
    target = torch.full_like(v0, 0.5, dtype=torch.float64)
    xT = runtime.RolloutFunction.apply(v0, Pd, mesh, prm, 5, 2, ctx=ctx)
    loss = ((xT - target) ** 2).sum()
    loss.backward()
    seeds = {"x": (2 * (xT.detach() - target)).cpu().numpy(), "v": np.zeros((3, P.n)), "F": np.zeros((9, P.n))}
    ref, _, _ = tape_grad(tb, ctx, mesh, P, prm, 5, 2, seeds)
    assert rel_l2(v0.grad.cpu().numpy(), ref["v"]) <= 1e-12


def test_rollout_grad_centre_of_mass(tb, ctx):
    """The differentiable-rollout loss (squared distance of the final centre of
    mass to a target) on a small sphere: with no walls the centre of mass moves
    as sum_i m_i v_i / M, so dL/dv0_p = 2 (x_com - c) T m_p / M to first order."""
    from tesserae_b200 import runtime
    sc = tb.scenes.sphere3d(scale=8)
    P = sc.particles
    Pd = P.to("torch", device="cuda", dtype=np.float32)
    c = torch.tensor(sc.meta["target"], dtype=torch.float64, device="cuda")[:, None]
    nsteps = 40

    def loss_grad(Q):
        xcom = Q.x.double().mean(dim=1, keepdim=True)
        r = xcom - c
        return float((r ** 2).sum()), (2 * r / Q.n).expand(-1, Q.n).contiguous(), torch.zeros_like(Q.v,
                                                                                                   dtype=torch.float64)

    loss, gv, glogE = runtime.rollout_grad(Pd, sc.mesh, sc.params, nsteps, loss_grad, checkpoint_every=10, ctx=ctx)
    xcom = P.x.mean(axis=1, keepdims=True) + nsteps * sc.params.dt * P.v.mean(axis=1, keepdims=True)
    expect = 2 * (xcom - np.array(sc.meta["target"])[:, None]) * nsteps * sc.params.dt / P.n
    assert rel_l2(gv.cpu().numpy(), np.broadcast_to(expect, P.v.shape)) <= 1e-3
    assert glogE is not None and torch.isfinite(glogE).all()


def x64_tape_grad(tb, ctx, mesh, P, prm, nsteps, every, seeds, x64=True):
    """Gradients of the mixed FP32 form's tape, with FP64 positions (x64) or FP32 ones."""
    from tesserae_b200 import runtime
    Pd = P.to("torch", device="cuda", dtype=np.float32, x64=x64)
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(mesh, np.float32, backend="torch", device="cuda")
    runtime.tape_forward(G, Pd, part, mesh, prm, nsteps, every, ctx=ctx)
    adj = device_adjoint(tb, P, seeds)
    runtime.tape_backward(G, Pd, part, mesh, prm, adj, ctx=ctx)
    ctx.synchronize()
    return adj.numpy(), Pd.to("numpy")


@pytest.mark.parametrize("every", [3, 1])
@pytest.mark.parametrize("case", ["bspline3d", "ugimp", "fluid", "walls"])
def test_x64_tape_close_to_fp64(tb, oracle, ctx, case, every):
    """The FP64-position form's tape against the FP64 oracle's rollout gradient:
    within 2e-6 relative L2 per field (measured 5e-9 to 3e-7), and at most half
    the FP32-position tape's error (whose positions round to FP32 every step;
    measured 4 to 15 times larger)."""
    mesh, P, prm = box_scene(tb, **CASES[case])
    nsteps = 7
    seeds = random_seeds(P, np.random.default_rng(11))
    ref, _ = oracle_rollout_grad(tb, oracle, mesh, P, prm, nsteps, seeds)
    got, restored = x64_tape_grad(tb, ctx, mesh, P, prm, nsteps, every, seeds)
    f32, _ = x64_tape_grad(tb, ctx, mesh, P, prm, nsteps, every, seeds, x64=False)
    assert np.array_equal(restored.x, P.x)  # the step-0 FP64 positions are back
    for k in ("x", "v", "F", "mu", "lam"):
        e64, e32 = rel_l2(got[k], getattr(ref, k)), rel_l2(f32[k], getattr(ref, k))
        print(f"x64 tape {case} every={every} {k}: {e64:.3g} (FP32 positions {e32:.3g})")
        assert e64 <= 2e-6, (case, k, e64)
        assert e64 <= 0.5 * e32 + 1e-9, (case, k, e64, e32)


def test_x64_adjoint_step_matches_oracle(tb, oracle, ctx):
    """One reverse step of the FP64-position form against the FP64 oracle's."""
    from tesserae_b200 import runtime
    mesh, P, prm = box_scene(tb, dim=3)
    seeds = random_seeds(P, np.random.default_rng(12))
    adj_o = host_adjoint(tb, P, seeds)
    oracle.adjoint_step(mesh, P, tb.generate_grid(mesh, np.float64), prm, adj_o)
    Pd = P.to("torch", device="cuda", dtype=np.float32, x64=True)
    adj_d = device_adjoint(tb, P, seeds)
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(mesh, np.float32, backend="torch", device="cuda")
    runtime.adjoint_step(G, Pd, part, mesh, prm, adj_d, ctx=ctx)
    ctx.synchronize()
    got = adj_d.numpy()
    for k in ("x", "v", "F", "mu", "lam"):
        assert rel_l2(got[k], getattr(adj_o, k)) <= 1e-4, (k, rel_l2(got[k], getattr(adj_o, k)))
