"""The oracle's von Mises model (the Taylor impact's `vonmises_model`,
docs/src/gpu.md:362-391) against an independent numpy restatement that uses
numpy.linalg.eigh for the spectral decomposition. A G2P over a grid at rest
leaves dF = I, so it applies the model to the particle's F as given: elastic
and plastic particles, first yield and re-yield with hardening."""
import numpy as np

from helpers import rel_l2

SYM = [(0, 0), (1, 0), (2, 0), (1, 1), (2, 1), (2, 2)]  # Tensorial symmetric order 11,21,31,22,32,33


def vonmises_np(Cp, ep, F, lam, mu, H, ty0):
    kappa = lam + 2.0 * mu / 3.0
    J = np.linalg.det(F)
    p = kappa * np.log(J) / J
    b = F @ Cp @ F.T
    b = 0.5 * (b + b.T)
    vals, vecs = np.linalg.eigh(b)
    lst = np.sqrt(vals)
    tau_tr = 2.0 * mu * np.log(lst) - 2.0 * mu / 3.0 * np.log(J)
    nrm = np.sqrt(1.5 * np.dot(tau_tr, tau_tr))
    f = nrm - (ty0 + H * ep)
    if f > 0:
        dg = f / (3.0 * mu + H)
        deps = dg * 1.5 * tau_tr / nrm
        le = np.exp(np.log(lst) - deps)
        tau = tau_tr - 2.0 * mu * deps
    else:
        dg, le, tau = 0.0, lst, tau_tr
    be = vecs @ np.diag(le ** 2) @ vecs.T
    sig = vecs @ np.diag(tau / J + p) @ vecs.T
    Fi = np.linalg.inv(F)
    C = Fi @ be @ Fi.T
    return sig, 0.5 * (C + C.T), ep + dg


def test_vonmises_model_matches_numpy(tb, oracle):
    rng = np.random.default_rng(11)
    n = 64
    mesh = tb.CartesianMesh(0.1, (0.0, 1.0), (0.0, 1.0), (0.0, 1.0))
    P = tb.Particles(n, 3, optional=("eps_p", "Cp_inv"))
    P.x[...] = rng.uniform(0.3, 0.7, size=(3, n))
    P.V[...] = 1e-3
    E, nu = 117e9, 0.35
    lam, mu = E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))
    H, ty0 = 0.1e9, 0.4e9
    Fs, Cps, eps = [], [], []
    for i in range(n):
        scale = [1e-4, 3e-3, 2e-2][i % 3]  # elastic, near yield, well past yield
        F = np.eye(3) + rng.normal(0.0, scale, size=(3, 3))
        A = np.eye(3) + rng.normal(0.0, 0.01 * (i % 2), size=(3, 3))  # some particles yielded before
        Cp = np.linalg.inv(A.T @ A)
        ep = 0.0 if i % 2 == 0 else rng.uniform(0.0, 0.05)
        Fs.append(F), Cps.append(Cp), eps.append(ep)
        for r in range(3):
            for c in range(3):
                P.F[r + 3 * c, i] = F[r, c]
        for k, (r, c) in enumerate(SYM):
            P.Cp_inv[k, i] = Cp[r, c]
        P.eps_p[i] = ep
    G = tb.generate_grid(mesh)
    prm = tb.step_params(1e-8, mass=1.0, V0=1e-3, mu=mu, lam=lam, material=tb._abi.MATERIAL_VONMISES,
                         hardening=H, yield_stress=ty0)
    oracle.g2p(mesh, G, P, prm)
    yielded = 0
    for i in range(n):
        sig, Cpn, epn = vonmises_np(Cps[i], eps[i], Fs[i], lam, mu, H, ty0)
        got_sig = np.zeros((3, 3))
        got_C = np.zeros((3, 3))
        for k, (r, c) in enumerate(SYM):
            got_sig[r, c] = got_sig[c, r] = P.sigma[k, i]
            got_C[r, c] = got_C[c, r] = P.Cp_inv[k, i]
        assert rel_l2(got_sig, sig) <= 1e-9, (i, rel_l2(got_sig, sig))
        assert rel_l2(got_C, Cpn) <= 1e-12, i
        assert abs(P.eps_p[i] - epn) <= 1e-12 * max(1.0, epn), i
        assert P.V[i] == 1e-3  # det(dF) = 1
        yielded += epn > eps[i]
    assert yielded >= n // 4  # the plastic branch ran
