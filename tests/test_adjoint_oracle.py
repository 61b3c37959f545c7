"""The oracle's reverse step against central finite differences of the oracle's
own FP64 forward rollout (CPU only).

Directional derivatives of a linear loss on the final state (random weights on
x, v and F) with respect to the initial x, v, F and the per-particle Lame
parameters must match central differences to 1e-6 relative. The FP64 forward
makes the difference quotient accurate to about 1e-8 with eps chosen per field:
1e-7 for x (nodes that a window just entered carry tiny masses, so the loss
curves sharply in x there and 1e-6 is already too coarse for uGIMP), 1e-6 for
v and F, 1e-5 (relative) for the Lame parameters, whose small sensitivities
would drown in the rounding of the loss at smaller steps. The kernels are C1,
so nothing but an error in the hand-written adjoint moves the two apart by more.
"""
import numpy as np
import pytest

from adjoint_helpers import (box_scene, directional, linear_loss, oracle_rollout, oracle_rollout_grad, perturbed,
                             random_seeds)

CASES = {
    "bspline3d": dict(dim=3),
    "pic_blend": dict(dim=3, alpha=0.9),
    "ugimp": dict(dim=3, basis=1),
    "fluid": dict(dim=3, material=1, E=1e3),
    "walls": dict(dim=3, lo=0.02, hi=0.4, walls=0b111111),
    "bspline2d": dict(dim=2, cells=16),
}


def scales(P, field):
    if field in ("mu", "lam"):
        return getattr(P, field).astype(np.float64)
    return 1.0


@pytest.mark.parametrize("case", sorted(CASES))
def test_oracle_adjoint_matches_finite_differences(tb, oracle, case):
    mesh, P, prm = box_scene(tb, **CASES[case])
    nsteps = 4
    rng = np.random.default_rng(11)
    seeds = random_seeds(P, rng)
    adj, _ = oracle_rollout_grad(tb, oracle, mesh, P, prm, nsteps, seeds)
    for field, eps in (("x", 1e-7), ("v", 1e-6), ("F", 1e-6), ("mu", 1e-5), ("lam", 1e-5)):
        shape = getattr(P, field).shape
        delta = rng.normal(size=shape) * scales(P, field)
        Lp = linear_loss(oracle_rollout(tb, oracle, mesh, perturbed(P, prm, field, delta, eps), prm, nsteps), seeds)
        Lm = linear_loss(oracle_rollout(tb, oracle, mesh, perturbed(P, prm, field, delta, -eps), prm, nsteps), seeds)
        fd = (Lp - Lm) / (2 * eps)
        ad = directional(adj, field, delta)
        assert abs(ad - fd) <= 1e-6 * max(abs(fd), 1e-3), (case, field, ad, fd)


def test_adjoint_rejects_unsupported(tb, oracle):
    """APIC needs the B sensitivity array; the von Mises model has no adjoint."""
    mesh, P, prm = box_scene(tb, dim=3)
    prm.transfer = tb._abi.TB_TRANSFER_APIC
    adj = tb.Adjoint(P.n, 3)
    with pytest.raises(RuntimeError):
        oracle.adjoint_step(mesh, P, tb.generate_grid(mesh, np.float64), prm, adj)
    prm.transfer = tb._abi.TB_TRANSFER_FLIP
    prm.material = tb._abi.MATERIAL_VONMISES
    with pytest.raises(RuntimeError):
        oracle.adjoint_step(mesh, P, tb.generate_grid(mesh, np.float64), prm, adj)
