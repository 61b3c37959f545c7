"""The oracle's @P2G / @G2P against the reference test's own hand-written
loops (test/transfer.jl:61-133, restated in tests/transfer_fixture.py) on the
reference's deterministic fixture state: an independent second statement of
the transfer semantics (gravity term, -V sigma grad w, the m != 0 guard of the
grid half, the PIC/FLIP blend, grad v, the position and F updates).

The reference compares with `isapprox` (rtol sqrt(eps)); these compare to
1e-12 relative to the field's scale, both sides being FP64 sums of the same
terms in different orders."""
import numpy as np
import pytest

import transfer_fixture as fx

DT, GRAVITY, ALPHA = 0.01, (0.0, -9.81), 0.95


def cases(tb):
    # the reference fixture mesh (every window truncated at h = 1 on (0,2)^2)
    yield "fixture", tb.CartesianMesh(1.0, (0.0, 2.0), (0.0, 2.0)), None, True
    # full windows only: the manual PIC/FLIP loop and the @G2P body agree
    yield "interior", tb.CartesianMesh(1.0, (0.0, 8.0), (0.0, 8.0)), \
        (lambda x: np.all((x >= 1.5) & (x <= 6.5), axis=0)), False
    # a finer mesh with interior and truncated windows
    yield "mixed", tb.CartesianMesh(0.25, (0.0, 2.0), (0.0, 1.5)), None, True


def params(tb):
    return tb.step_params(DT, mass=0.0, gravity=GRAVITY, flip_alpha=ALPHA, mu=1.0, lam=1.0)


def scale(a):
    return max(float(np.max(np.abs(a))), 1e-300)


@pytest.mark.parametrize("name", ["fixture", "interior", "mixed"])
def test_p2g_matches_manual_loops(tb, oracle, name):
    mesh, keep, _ = next((m, k, t) for n, m, k, t in cases(tb) if n == name)
    P = fx.initialize_state(tb, mesh, keep=keep)
    prm = params(tb)
    W = fx.weights_of(tb, oracle, mesh, P, prm)
    ref = fx.manual_p2g(mesh, P, W, DT, GRAVITY)
    G = tb.generate_grid(mesh)
    G.m[...] = 1.0  # initialize_mpm_state! sets the grid; assigned targets are zeroed by @P2G
    G.mv[...] = 0.3
    G.f[...] = -0.7
    oracle.p2g(mesh, P, G, prm)
    oracle.grid_update(mesh, G, prm)
    for k in ("m", "mv", "f", "vn", "v"):
        got = getattr(G, k)
        assert np.max(np.abs(got - ref[k])) <= 1e-12 * scale(ref[k]), (name, k)


@pytest.mark.parametrize("name", ["fixture", "interior", "mixed"])
def test_g2p_matches_manual_loops(tb, oracle, name):
    mesh, keep, truncated = next((m, k, t) for n, m, k, t in cases(tb) if n == name)
    P = fx.initialize_state(tb, mesh, keep=keep)
    prm = params(tb)
    W = fx.weights_of(tb, oracle, mesh, P, prm)
    grid = fx.manual_p2g(mesh, P, W, DT, GRAVITY)
    # the manual loop's blend (1 - a) sum w v_i + a (v_p + sum w (v_i - vn_i));
    # with full windows the @G2P body of the test gives the same result
    forms = [False] if truncated else [False, True]
    refs = [fx.manual_g2p(mesh, P, W, grid, ALPHA, DT, macro_form=f) for f in forms]
    G = tb.generate_grid(mesh)
    G.v[...] = grid["v"]
    G.vn[...] = grid["vn"]
    Q = P.to("numpy")
    oracle.g2p(mesh, G, Q, prm)
    for ref in refs:
        for k in ("v", "grad_v", "x", "F"):
            got = getattr(Q, k)
            assert np.max(np.abs(got - ref[k])) <= 1e-12 * scale(ref[k]), (name, k)


def test_fixture_state_is_the_reference_one(tb):
    """The first particle of the reference fixture: x = (0.25, 0.25) on
    CartesianMesh(1.0, (0,2), (0,2)) with GridSampling(), p = 1."""
    mesh = tb.CartesianMesh(1.0, (0.0, 2.0), (0.0, 2.0))
    P = fx.initialize_state(tb, mesh)
    assert P.n == 16
    assert list(P.x[:, 0]) == [0.25, 0.25]
    assert np.isclose(P.m[0], 1.05) and np.isclose(P.V[0], 0.21)
    assert np.allclose(P.v[:, 0], [0.17, -0.235])
    assert np.allclose(P.F[:, 0], [1.002, 0.0, 0.0, 0.999])
