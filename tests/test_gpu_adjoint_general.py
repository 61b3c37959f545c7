"""The general device reverse step (WLS and KernelCorrection bases, APIC; the
particle-parallel kernels with Dual3 weight derivatives) through the C ABI
against the oracle's general reverse step, which tests/test_adjoint_general.py
pins to forward-mode dual numbers: one step (FP64 to 1e-10 relative L2 per
field, the mixed FP32 form to 1e-4) and the checkpointed tape over several
steps (FP64 to 1e-9), including the APIC matrix sensitivity."""
import numpy as np
import pytest

from helpers import rel_l2
from test_adjoint_general import CASES, rollout_grad, scene

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def seeds_for(P, apic, rng):
    outs = ("x", "v", "F", "B") if apic else ("x", "v", "F")
    return {k: rng.normal(size=getattr(P, k).shape) for k in outs}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-10), (np.float32, 1e-4)])
def test_general_adjoint_step_matches_oracle(tb, oracle, ctx, case, dtype, tol):
    from tesserae_b200 import runtime
    mesh, P, prm = scene(tb, **CASES[case])
    P = P.to("numpy", dtype=dtype)
    apic = prm.transfer == 1
    seeds = seeds_for(P, apic, np.random.default_rng(5))
    adj_o = tb.Adjoint(P.n, P.dim, apic=apic)
    for k, v in seeds.items():
        getattr(adj_o, k)[...] = v
    oracle.adjoint_step(mesh, P, tb.generate_grid(mesh, dtype), prm, adj_o)
    adj_d = tb.Adjoint(P.n, P.dim, backend="torch", device="cuda", apic=apic)
    for k, v in seeds.items():
        getattr(adj_d, k).copy_(torch.from_numpy(v))
    runtime.adjoint_step(tb.generate_grid(mesh, dtype, backend="torch", device="cuda"), P.to("torch", device="cuda"),
                         tb.Partition(mesh, P.n, backend="torch", device="cuda"), mesh, prm, adj_d, ctx=ctx)
    ctx.synchronize()
    got = adj_d.numpy()
    for k in ("x", "v", "F", "mu", "lam") + (("B",) if apic else ()):
        err = rel_l2(got[k], getattr(adj_o, k))
        assert err <= tol, (case, k, err)


@pytest.mark.parametrize("every", [2, 1])  # 1: the whole tape
@pytest.mark.parametrize("case", ["dambreak_set", "apic_bspline", "wls_bspline"])
def test_general_tape_matches_oracle_rollout(tb, oracle, ctx, case, every):
    from tesserae_b200 import runtime
    mesh, P, prm = scene(tb, **CASES[case])
    apic = prm.transfer == 1
    nsteps = 5
    seeds = seeds_for(P, apic, np.random.default_rng(7))
    adj_o, final = rollout_grad(tb, oracle, mesh, P, prm, nsteps, seeds, apic)
    Pd = P.to("torch", device="cuda")
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(mesh, np.float64, backend="torch", device="cuda")
    runtime.tape_forward(G, Pd, part, mesh, prm, nsteps, every, ctx=ctx)
    ctx.synchronize()
    assert rel_l2(Pd.x.cpu().numpy(), final.x) <= 1e-12
    adj_d = tb.Adjoint(P.n, P.dim, backend="torch", device="cuda", apic=apic)
    for k, v in seeds.items():
        getattr(adj_d, k).copy_(torch.from_numpy(v))
    runtime.tape_backward(G, Pd, part, mesh, prm, adj_d, ctx=ctx)
    ctx.synchronize()
    got = adj_d.numpy()
    for k in ("x", "v", "F", "mu", "lam") + (("B",) if apic else ()):
        err = rel_l2(got[k], getattr(adj_o, k))
        assert err <= 1e-9, (case, k, err)


@pytest.mark.parametrize("case", ["dambreak_set", "apic_bspline", "wls_bspline"])
def test_general_x64_tape_close_to_fp64(tb, oracle, ctx, case):
    """The FP64-position form's tape on the general reverse step (WLS, APIC,
    fluid) against the FP64 oracle's rollout gradient: within 2e-6 relative L2
    (measured 2e-9 to 3e-7)."""
    from tesserae_b200 import runtime
    mesh, P, prm = scene(tb, **CASES[case])
    if P.dim != 3:
        pytest.skip("the FP64-position form runs WLS and APIC in 3D only")
    apic = prm.transfer == 1
    nsteps = 5
    seeds = seeds_for(P, apic, np.random.default_rng(9))
    adj_o, _ = rollout_grad(tb, oracle, mesh, P, prm, nsteps, seeds, apic)
    Pd = P.to("torch", device="cuda", dtype=np.float32, x64=True)
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(mesh, np.float32, backend="torch", device="cuda")
    runtime.tape_forward(G, Pd, part, mesh, prm, nsteps, 1, ctx=ctx)
    adj_d = tb.Adjoint(P.n, P.dim, backend="torch", device="cuda", apic=apic)
    for k, v in seeds.items():
        getattr(adj_d, k).copy_(torch.from_numpy(v))
    runtime.tape_backward(G, Pd, part, mesh, prm, adj_d, ctx=ctx)
    ctx.synchronize()
    got = adj_d.numpy()
    for k in ("x", "v", "F", "mu", "lam") + (("B",) if apic else ()):
        err = rel_l2(got[k], getattr(adj_o, k))
        print(f"x64 general tape {case} {k}: {err:.3g}")
        assert err <= 2e-6, (case, k, err)
