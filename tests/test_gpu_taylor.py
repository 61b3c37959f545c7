"""The Taylor impact path (docs/src/gpu.md:202-392) on the device against the
oracle: KernelCorrection(BSpline(Quadratic())) weights (a rod standing on the
mesh floor, so every step has truncated windows), the von Mises model with its
plastic state, V = det(dF) V, the slip floor of one node layer, and the
adaptive time step's wave speed. The scene is the Taylor impact at 4x the
spacing (22 954 particles).

Tolerances: FP64 step against the FP64 oracle <= 1e-9 relative L2 per field
after 20 steps (sums in another order); FP32 forms <= 1e-4 on x, v and F,
<= 1e-3 on sigma (a stress of order the yield stress built from F, whose
FP32 rounding it amplifies by E / sigma_y ~ 300); the wave speed to 1e-12.
"""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

FIELDS = ("x", "v", "F", "V", "sigma", "Cp_inv", "eps_p")


def scene(tb):
    return tb.scenes.taylor3d(scale=4)


def run_device(tb, ctx, sc, dtype, x64, nsteps):
    from tesserae_b200 import runtime
    P = sc.particles.to("torch", device="cuda", dtype=dtype, x64=x64)
    part = tb.Partition(sc.mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(sc.mesh, dtype, backend="torch", device="cuda")
    runtime.step(G, P, part, sc.mesh, sc.params, nsteps, ctx=ctx)
    ctx.synchronize()
    return P.numpy()


@pytest.fixture(scope="module")
def oracle20(tb, oracle):
    sc = scene(tb)
    P = sc.particles.to("numpy")
    G = tb.generate_grid(sc.mesh)
    oracle.step(sc.mesh, P, G, sc.params, 20)
    return P.numpy()


def test_taylor_fp64_matches_oracle(tb, ctx, oracle20):
    sc = scene(tb)
    got = run_device(tb, ctx, sc, np.float64, False, 20)
    for k in FIELDS:
        assert rel_l2(got[k], oracle20[k]) <= 1e-9, (k, rel_l2(got[k], oracle20[k]))
    assert np.max(oracle20["eps_p"]) > 0.0  # the rod yields at the floor within 20 steps


@pytest.mark.parametrize("x64", [False, True])
def test_taylor_fp32_forms_match_oracle(tb, ctx, oracle20, x64):
    sc = scene(tb)
    got = run_device(tb, ctx, sc, np.float32, x64, 20)
    for k, tol in (("x", 1e-4), ("v", 1e-4), ("F", 1e-4), ("V", 1e-4), ("sigma", 1e-3), ("Cp_inv", 1e-4)):
        assert rel_l2(got[k], oracle20[k]) <= tol, (k, x64, rel_l2(got[k], oracle20[k]))


def test_taylor_floor_stops_the_rod(tb, ctx):
    """After 60 steps (about 3.7 us at 4x the spacing) the bottom of the rod has
    stopped on the floor: the particles within one cell of it move downwards at
    well under the impact speed, and none has gone through the floor."""
    sc = scene(tb)
    got = run_device(tb, ctx, sc, np.float64, False, 60)
    h = sc.mesh.h
    near = got["x"][2] < h
    assert near.any()
    assert np.all(got["x"][2] > -0.5 * h)
    assert np.mean(-got["v"][2][near]) < 0.5 * 227.0


def test_max_wave_speed(tb, ctx):
    from tesserae_b200 import runtime
    sc = scene(tb)
    P = sc.particles
    P.v[0] = np.linspace(-3.0, 5.0, P.n)  # not every particle at the same speed
    prm = sc.params
    want = np.max(np.sqrt((prm.lambda_ + 2 * prm.mu) / (prm.mass / P.V)) + np.linalg.norm(P.v, axis=0))
    for dtype in (np.float64, np.float32):
        got = runtime.max_wave_speed(P.to("torch", device="cuda", dtype=dtype), prm, ctx=ctx)
        assert got == pytest.approx(want, rel=1e-12 if dtype == np.float64 else 1e-6), dtype


def test_adaptive_steps_follow_the_cfl_rule(tb, ctx):
    from tesserae_b200 import runtime
    sc = scene(tb)
    P = sc.particles.to("torch", device="cuda")
    part = tb.Partition(sc.mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(sc.mesh, backend="torch", device="cuda")
    t1 = runtime.adaptive_steps(G, P, part, sc.mesh, sc.params, 1, ctx=ctx)
    assert t1 == pytest.approx(sc.params.dt, rel=1e-12)  # the first step's dt is the scene's
    host = P.numpy()
    dt2 = tb.scenes.taylor_dt(host["v"], host["V"], sc.params.mass, sc.params.mu, sc.params.lambda_, sc.mesh.h)
    t2 = runtime.adaptive_steps(G, P, part, sc.mesh, sc.params, 1, ctx=ctx)
    assert t2 == pytest.approx(dt2, rel=1e-12)
