"""The reference's own transfer test fixture and its hand-written loops,
restated in numpy: a second, independent statement of the @P2G / @G2P
semantics that pins the oracle's transfer layer (and, on the GPU, the
kernels) to what Tesserae.jl's tests require.

  initialize_mpm_state!   test/transfer.jl:61-83   deterministic particle state
  manual_p2g!             test/transfer.jl:85-109  m, mv, f (gravity, -V sigma grad w), grid half
  manual_g2p_pic_flip!    test/transfer.jl:111-133 PIC/FLIP blend, grad v, x, F
  @G2P body               test/transfer.jl:254-259 the macro form the kernels implement

The reference fixture (test/transfer.jl:3-29) samples CartesianMesh(1.0, (0,2),
(0,2)) with GridSampling() and uses BSpline(Linear()); this path has no linear
B-spline, so the same state is put on quadratic B-spline weights (stored
weights from tb_update_weights, whose values are pinned by the reference's
basis known answers). The loops are basis-agnostic: they only read the stored
w, grad w and window of each particle.
"""
from __future__ import annotations

import numpy as np


def initialize_state(tb, mesh, alg=None, keep=None):
    """Particles of generate_particles(mesh; alg=GridSampling()) with the state
    of initialize_mpm_state! (test/transfer.jl:62-70), p the 1-based particle
    index after the optional `keep` filter. Returns a host FP64 Particles with
    per-particle mass."""
    pts = tb.generate_points(alg or tb.GridSampling(), mesh)
    if keep is not None:
        pts = pts[:, keep(pts)]
    n = pts.shape[1]
    P = tb.Particles(n, 2, np.float64, optional=("m",))
    P.x[...] = pts
    p = np.arange(1, n + 1, dtype=np.float64)
    P.m[...] = 1.0 + 0.05 * p
    P.V[...] = 0.2 + 0.01 * p
    P.v[0] = 0.15 + 0.02 * p
    P.v[1] = -0.25 + 0.015 * p
    P.F[...] = 0.0
    P.F[0] = 1.0 + 0.002 * p  # diagm(Vec(1 + 0.002p, 1 - 0.001p)), column-major (11, 21, 12, 22)
    P.F[3] = 1.0 - 0.001 * p
    # sigma = symmetric(a (x) b), a = (1 + 0.03p, 0.2), b = (0.4, 0.8 + 0.01p); stored (11, 21, 22)
    a1, a2, b1, b2 = 1.0 + 0.03 * p, 0.2, 0.4, 0.8 + 0.01 * p
    P.sigma[0] = a1 * b1
    P.sigma[1] = 0.5 * (a1 * b2 + a2 * b1)
    P.sigma[2] = a2 * b2
    return P


def weights_of(tb, oracle, mesh, P, params):
    """Stored weights (w, grad w, window) per particle from the oracle."""
    W = tb.generate_basis_weights(mesh.dim, P.n)
    oracle.update_weights(mesh, P, params, W)
    return W


def _nodes(mesh, W, p):
    """(slot, linear node index) pairs of particle p's window; slot s = i + 3 j."""
    win = W.window[p]
    out = []
    for j in range(win[2] - 1, win[3]):
        for i in range(win[0] - 1, win[1]):
            s = (i - (win[0] - 1)) + 3 * (j - (win[2] - 1))
            out.append((s, i + mesh.n_nodes[0] * j))
    return out


def sym2(sig, p):
    return np.array([[sig[0][p], sig[1][p]], [sig[1][p], sig[2][p]]])


def manual_p2g(mesh, P, W, dt, gravity):
    """manual_p2g! (test/transfer.jl:85-109): returns m, mv, f, vn, v (FP64)."""
    N = mesh.nnodes
    m = np.zeros(N)
    mv = np.zeros((2, N))
    f = np.zeros((2, N))
    g = np.asarray(gravity, dtype=np.float64)
    for p in range(P.n):
        vp = P.v[:, p]
        S = sym2(P.sigma, p)
        for s, i in _nodes(mesh, W, p):
            w = W.w[p, s]
            dw = W.grad_w[p, s]
            m[i] += w * P.m[p]
            mv[:, i] += w * P.m[p] * vp
            f[:, i] += w * P.m[p] * g
            f[:, i] -= P.V[p] * (S @ dw)
    minv = np.where(m != 0, 1.0 / np.where(m != 0, m, 1.0), 0.0)
    vn = mv * minv
    v = vn + (f * minv) * dt
    return {"m": m, "mv": mv, "f": f, "vn": vn, "v": v}


def manual_g2p(mesh, P, W, grid, alpha, dt, macro_form=False):
    """manual_g2p_pic_flip! (test/transfer.jl:111-133), or with `macro_form` the
    @G2P body of test/transfer.jl:254-259 (v_p = sum w ((1-a) v_i + a (v_p +
    v_i - vn_i)); the two agree where the weights sum to one). Returns v, grad_v
    (column-major 11, 21, 12, 22), x, F."""
    n = P.n
    v_out = np.zeros((2, n))
    gv = np.zeros((4, n))
    x = P.x.copy()
    F = np.zeros((4, n))
    for p in range(n):
        vpic = np.zeros(2)
        dflip = np.zeros(2)
        L = np.zeros((2, 2))
        dx = np.zeros(2)
        wsum = 0.0
        for s, i in _nodes(mesh, W, p):
            w = W.w[p, s]
            dw = W.grad_w[p, s]
            vi, vni = grid["v"][:, i], grid["vn"][:, i]
            vpic += w * vi
            dflip += w * (vi - vni)
            L += np.outer(vi, dw)
            dx += w * vi * dt
            wsum += w
        vp = P.v[:, p]
        if macro_form:
            v_out[:, p] = (1 - alpha) * vpic + alpha * (wsum * vp + dflip)
        else:
            v_out[:, p] = (1 - alpha) * vpic + alpha * (vp + dflip)
        gv[:, p] = L.reshape(-1, order="F")
        x[:, p] += dx
        Fp = P.F[:, p].reshape(2, 2, order="F")
        F[:, p] = ((np.eye(2) + L * dt) @ Fp).reshape(-1, order="F")
    return {"v": v_out, "grad_v": gv, "x": x, "F": F}
