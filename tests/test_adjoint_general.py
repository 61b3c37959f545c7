"""The oracle's general reverse step (WLS and KernelCorrection bases, the APIC
transfer, the fluid; position derivatives of the weights from the weights in
dual numbers) against forward-mode derivatives of the same FP64 step
(tbo_step_dual), 1e-9 relative, for a linear loss on the final x, v, F and
(APIC) B. The WLS(uGIMP) + APIC + fluid + walls case is the dam-break
configuration's equation set."""
import numpy as np
import pytest

from adjoint_helpers import box_scene
from test_adjoint_dual import state_seeds

CASES = {
    "apic_bspline": dict(transfer=1),
    "apic_ugimp": dict(transfer=1, basis=1),
    "wls_bspline": dict(basis=2),
    "wls_ugimp": dict(basis=3),
    "kc_bspline_walls": dict(basis=4, lo=0.02, hi=0.4, walls=0b111111),
    "dambreak_set": dict(transfer=1, basis=3, material=1, E=1e3, lo=0.02, hi=0.4, walls=0b111111),
    "apic_2d": dict(transfer=1, dim=2, cells=16),
}


def scene(tb, transfer=0, **kw):
    mesh, P, prm = box_scene(tb, **kw)
    prm.transfer = transfer
    if transfer == 1:
        Q = P.to("numpy")
        opt = ("mu", "lam", "B")
        R = tb.Particles(Q.n, Q.dim, np.float64, optional=opt)
        for k in Q.FIELDS:
            if getattr(Q, k) is not None:
                getattr(R, k)[...] = getattr(Q, k)
        rng = np.random.default_rng(3)
        R.B[...] = rng.normal(0.0, 0.05, size=R.B.shape)
        P = R
    return mesh, P, prm


def rollout_grad(tb, oracle, mesh, P, prm, nsteps, seeds, apic):
    states = [P.to("numpy")]
    G = tb.generate_grid(mesh, np.float64)
    for _ in range(nsteps):
        Q = states[-1].to("numpy")
        oracle.step(mesh, Q, G, prm, 1)
        states.append(Q)
    adj = tb.Adjoint(P.n, P.dim, apic=apic)
    for k in seeds:
        getattr(adj, k)[...] = seeds[k]
    for s in reversed(range(nsteps)):
        oracle.adjoint_step(mesh, states[s], G, prm, adj)
    return adj, states[-1]


@pytest.mark.parametrize("case", sorted(CASES))
def test_general_reverse_step_matches_forward_mode(tb, oracle, case):
    mesh, P, prm = scene(tb, **CASES[case])
    apic = prm.transfer == 1
    nsteps = 3
    rng = np.random.default_rng(29)
    D, n = P.dim, P.n
    outs = ("x", "v", "F", "B") if apic else ("x", "v", "F")
    seeds = {k: rng.normal(size=getattr(P, k).shape) for k in outs}
    adj, final = rollout_grad(tb, oracle, mesh, P, prm, nsteps, seeds, apic)
    fields = ("x", "v", "F", "mu", "lam", "B") if apic else ("x", "v", "F", "mu", "lam")
    for field in fields:
        delta = rng.normal(size=getattr(P, field).shape)
        if field in ("mu", "lam"):
            delta = delta * getattr(P, field)
        val, der = oracle.directional_derivative(mesh, P, prm, nsteps, state_seeds(P, prm, field, delta),
                                                 outputs=outs)
        assert np.array_equal(val["x"], final.x)
        fwd = sum(float(np.sum(seeds[k] * der[k])) for k in outs)
        rev = float(np.sum(getattr(adj, field) * delta))
        assert abs(fwd - rev) <= 1e-9 * max(abs(fwd), 1e-6), (case, field, fwd, rev)
