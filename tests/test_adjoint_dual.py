"""The oracle's hand-written reverse step against forward-mode derivatives:
the same FP64 oracle step run in dual numbers (tbo_step_dual: every particle
and grid value carries one directional derivative through the binning, the
kernels' branches, P2G, the grid half, G2P and the constitutive update). This
is the gradient oracle that stands in for differentiating the reference with
ForwardDiff. Both sides are exact derivatives evaluated in FP64, so they agree
to rounding (1e-9 relative), far tighter than the finite differences of
tests/test_adjoint_oracle.py. Seeds of the stress and volume follow their
dependence on F, mu and lambda (sigma = sigma(F), V = V0 det F), taken by
complex-step differentiation of that closed form."""
import numpy as np
import pytest

from adjoint_helpers import box_scene, directional, neo_hookean, oracle_rollout_grad, random_seeds
from test_adjoint_oracle import CASES


def state_seeds(P, prm, field, delta):
    """Derivative seeds of every stored field for a perturbation `delta` of
    `field`, keeping sigma and V the functions of F, mu and lambda they are."""
    D, n = P.dim, P.n
    seed = {field: delta}
    if field in ("F", "mu", "lam"):
        h = 1e-30
        F = P.F.astype(np.complex128)
        mu = P.mu.astype(np.complex128)
        lam = P.lam.astype(np.complex128)
        if field == "F":
            F = F + 1j * h * delta
        elif field == "mu":
            mu = mu + 1j * h * delta
        else:
            lam = lam + 1j * h * delta
        sig, J = neo_hookean(F, mu, lam, prm.material)
        V0 = P.V0.astype(np.float64) if P.V0 is not None else np.full(n, prm.V0)
        dsig = np.zeros_like(P.sigma)
        k = 0
        for c in range(D):
            for r in range(c, D):
                dsig[k] = sig[:, r, c].imag / h
                k += 1
        seed["sigma"] = dsig
        seed["V"] = V0 * J.imag / h
    return seed


@pytest.mark.parametrize("case", sorted(CASES))
def test_reverse_step_matches_forward_mode(tb, oracle, case):
    mesh, P, prm = box_scene(tb, **CASES[case])
    nsteps = 4
    rng = np.random.default_rng(23)
    seeds = random_seeds(P, rng)
    adj, final = oracle_rollout_grad(tb, oracle, mesh, P, prm, nsteps, seeds)
    for field in ("x", "v", "F", "mu", "lam"):
        delta = rng.normal(size=getattr(P, field).shape)
        if field in ("mu", "lam"):
            delta = delta * getattr(P, field)
        val, der = oracle.directional_derivative(mesh, P, prm, nsteps, state_seeds(P, prm, field, delta),
                                                 outputs=("x", "v", "F"))
        # the dual rollout's values are the plain rollout's
        assert np.array_equal(val["x"], final.x) and np.array_equal(val["v"], final.v)
        fwd = sum(float(np.sum(seeds[k] * der[k])) for k in ("x", "v", "F"))
        rev = directional(adj, field, delta)
        assert abs(fwd - rev) <= 1e-9 * max(abs(fwd), 1e-6), (case, field, fwd, rev)
