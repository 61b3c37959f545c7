"""Shared pieces of the reverse-mode tests: small seeded scenes, consistent
initial stress, linear losses on the final state, and CPU rollouts (forward and
backward) through the oracle."""
import numpy as np


def neo_hookean(F, mu, lam, material):
    """sigma(F) (full, per particle) and J = det F for a (D*D, n) column-major F."""
    D = int(round(np.sqrt(F.shape[0])))
    n = F.shape[1]
    Fm = F.reshape(D, D, n).transpose(2, 1, 0)  # [p, r, c] = F[r + c D]
    J = np.linalg.det(Fm)
    eye = np.eye(D)[None]
    if material == 1:
        sig = (lam * (J - 1.0))[:, None, None] * eye
    else:
        B = Fm @ Fm.transpose(0, 2, 1)
        sig = (mu[:, None, None] * (B - eye) + (lam * np.log(J))[:, None, None] * eye) / J[:, None, None]
    return sig, J


def make_consistent(P, prm):
    """Set sigma and V from F (and mu, lambda, V0) so the state is the one the
    adjoint differentiates: sigma = sigma(F), V = V0 det F."""
    D, n = P.dim, P.n
    mu = P.mu.astype(np.float64) if P.mu is not None else np.full(n, prm.mu)
    lam = P.lam.astype(np.float64) if P.lam is not None else np.full(n, prm.lambda_)
    V0 = P.V0.astype(np.float64) if P.V0 is not None else np.full(n, prm.V0)
    sig, J = neo_hookean(P.F.astype(np.float64), mu, lam, prm.material)
    k = 0
    for c in range(D):
        for r in range(c, D):
            P.sigma[k] = sig[:, r, c]
            k += 1
    P.V[...] = V0 * J
    return P


def box_scene(tb, dim=3, cells=8, lo=0.25, hi=0.75, seed=0, material=0, basis=0, alpha=1.0, walls=0,
              E=1e3, nu=0.3, dt=1e-3, dtype=np.float64, vscale=0.5, gravity=None, ppc=2):
    """A box of particles (`ppc` per cell per axis, jittered, in lattice order)
    with random velocities and per-particle Lame parameters, on a unit-square/cube
    mesh."""
    rng = np.random.default_rng(seed)
    h = 1.0 / cells
    mesh = tb.CartesianMesh(h, *([(0.0, 1.0)] * dim))
    ax = np.arange(lo + h / (2 * ppc), hi, h / ppc)
    grids = np.meshgrid(*([ax] * dim), indexing="ij")
    pts = np.stack([g.ravel(order="F") for g in grids])
    pts = pts + rng.uniform(-h / (8 * ppc), h / (8 * ppc), size=pts.shape)
    n = pts.shape[1]
    P = tb.Particles(n, dim, np.float64, optional=("mu", "lam"))
    P.x[...] = pts
    P.v[...] = rng.uniform(-vscale, vscale, size=(dim, n))
    V0 = (h / ppc) ** dim
    mu, lam = tb.lame(E * np.exp(rng.normal(0.0, 0.1, size=n)), nu)
    P.mu[...] = mu
    P.lam[...] = lam
    if gravity is None:
        gravity = (0.0, 0.0, -9.81) if dim == 3 else (0.0, -9.81)
    prm = tb.step_params(dt, mass=1.0 * V0, V0=V0, mu=float(np.mean(mu)), lam=float(np.mean(lam)),
                         gravity=gravity, gimp_l=h / 2, flip_alpha=alpha, basis=basis, material=material,
                         wall_mask=walls, wall_layers=1 if walls else 0)
    make_consistent(P, prm)
    return mesh, P.to("numpy", dtype=dtype), prm


def linear_loss(P, seeds):
    """L = sum cx . x + cv . v + cF . F over the final state."""
    return float(np.sum(seeds["x"] * P.x.astype(np.float64)) + np.sum(seeds["v"] * P.v.astype(np.float64))
                 + np.sum(seeds["F"] * P.F))


def random_seeds(P, rng):
    D, n = P.dim, P.n
    return {"x": rng.normal(size=(D, n)), "v": rng.normal(size=(D, n)), "F": rng.normal(size=(D * D, n))}


def oracle_rollout(tb, oracle, mesh, P, prm, nsteps):
    Q = P.to("numpy")
    G = tb.generate_grid(mesh, P.dtype)
    oracle.step(mesh, Q, G, prm, nsteps)
    return Q


def oracle_rollout_grad(tb, oracle, mesh, P, prm, nsteps, seeds):
    """Reverse mode through `nsteps` oracle steps: the states are stored by a
    forward pass, then the oracle's adjoint step walks back over them."""
    states = [P.to("numpy")]
    G = tb.generate_grid(mesh, P.dtype)
    for _ in range(nsteps):
        Q = states[-1].to("numpy")
        oracle.step(mesh, Q, G, prm, 1)
        states.append(Q)
    adj = tb.Adjoint(P.n, P.dim)
    adj.x[...] = seeds["x"]
    adj.v[...] = seeds["v"]
    adj.F[...] = seeds["F"]
    for s in reversed(range(nsteps)):
        oracle.adjoint_step(mesh, states[s], G, prm, adj)
    return adj, states[-1]


def perturbed(P, prm, field, delta, eps):
    """Copy of P with `field` moved by eps * delta (sigma and V re-derived from F)."""
    Q = P.to("numpy")
    arr = getattr(Q, field)
    arr[...] = (arr.astype(np.float64) + eps * delta).astype(arr.dtype)
    make_consistent(Q, prm)
    return Q


def directional(adj, field, delta):
    key = {"x": "x", "v": "v", "F": "F", "mu": "mu", "lam": "lam"}[field]
    return float(np.sum(getattr(adj, key) * delta))
