"""The device @P2G / @G2P against the reference test's own hand-written loops
(test/transfer.jl:61-133, restated in tests/transfer_fixture.py) on the
reference's deterministic fixture state, through the C ABI: a check of the
kernels that does not go through the oracle's transfer code (only its stored
weights, pinned by the reference's basis known answers, feed the loops).
FP64 to 1e-12 and FP32 to 1e-5 of each field's scale."""
import numpy as np
import pytest

import transfer_fixture as fx
from test_transfer_fixture import ALPHA, DT, GRAVITY, cases, params, scale

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL = {np.float64: 1e-12, np.float32: 1e-5}


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("name", ["fixture", "interior", "mixed"])
def test_device_transfers_match_manual_loops(tb, ctx, oracle, name, dtype):
    from tesserae_b200 import runtime
    mesh, keep, _ = next((m, k, t) for n, m, k, t in cases(tb) if n == name)
    P = fx.initialize_state(tb, mesh, keep=keep)
    prm = params(tb)
    W = fx.weights_of(tb, oracle, mesh, P, prm)
    ref_g = fx.manual_p2g(mesh, P, W, DT, GRAVITY)
    ref_p = fx.manual_g2p(mesh, P, W, ref_g, ALPHA, DT)
    tol = TOL[dtype]

    Pd = P.to("torch", device="cuda", dtype=dtype)
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(mesh, dtype, backend="torch", device="cuda")
    G.m.fill_(1.0)  # stale grid values: assigned targets are zeroed by @P2G
    runtime.update(part, Pd, mesh, ctx=ctx)
    runtime.P2G(G, Pd, part, mesh, prm, ctx=ctx)
    ctx.synchronize()
    got = G.numpy()
    for k in ("m", "mv", "f", "vn", "v"):
        err = np.max(np.abs(got[k].astype(np.float64) - ref_g[k]))
        assert err <= tol * scale(ref_g[k]), (name, k, err)

    # G2P from the manual loops' grid
    G.v.copy_(torch.from_numpy(ref_g["v"].astype(dtype)))
    G.vn.copy_(torch.from_numpy(ref_g["vn"].astype(dtype)))
    runtime.G2P(G, Pd, mesh, prm, ctx=ctx)
    ctx.synchronize()
    got = Pd.numpy()
    for k in ("v", "grad_v", "x", "F"):
        err = np.max(np.abs(got[k].astype(np.float64) - ref_p[k]))
        assert err <= tol * scale(ref_p[k]), (name, k, err)
