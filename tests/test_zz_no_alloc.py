"""tb_bin_particles_noalloc: binning for callers that cannot allocate device
memory (no cudaMalloc, no tb_ctx), checked through the C ABI against the
allocating entry point tb_bin_particles_f32 / _f64 on two calls in a row (the
shared scratch keeps the previous call's contents). Bit-exact, like every
binning test. Collected last so a failure here leaves every other test run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def noalloc_bin(tb, mesh, P, precision):
    lib = tb._abi.load_library()
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    na, nass = C.c_int64(), C.c_int64()
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.tb_bin_particles_noalloc(C.byref(mesh.struct()), C.byref(P.struct()), precision,
                                      C.byref(part.struct()), C.c_void_p(stream), C.byref(na), C.byref(nass),
                                      err, 256)
    assert rc == tb._abi.TB_OK, err.value.decode()
    return part, (na.value, nass.value)


def allocating_bin(tb, ctx, mesh, P):
    from tesserae_b200 import runtime
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    runtime.update(part, P, mesh, ctx=ctx)
    return part, (part.nactive, part.nassigned)


@pytest.mark.parametrize("dtype,precision", [(np.float32, 1), (np.float64, 0)])
def test_noalloc_matches_allocating_binning_twice(tb, ctx, dtype, precision):
    rng = np.random.default_rng(42)
    mesh = tb.CartesianMesh(1 / 64, (0.0, 1.0), (0.0, 1.0), (0.0, 1.0))
    for call in range(2):
        # the second call has a different particle set and order than the first
        n = 300_000 if call == 0 else 123_457
        P = tb.Particles(n, 3, dtype)
        P.x[...] = rng.uniform(-0.02, 1.02, size=(3, n)).astype(dtype)
        if call == 1:
            P.x[:, : n // 2] = rng.uniform(0.3, 0.32, size=(3, n // 2)).astype(dtype)  # a crowded corner
        Pd = P.to("torch", device="cuda")
        a, ta = allocating_bin(tb, ctx, mesh, Pd)
        b, tb_ = noalloc_bin(tb, mesh, Pd, precision)
        assert ta == tb_
        na, nass = ta
        da, db = a.numpy(), b.numpy()
        for k in ("blockids", "counts", "offsets"):
            assert np.array_equal(da[k], db[k]), (call, k)
        assert np.array_equal(da["blocklist"][:na], db["blocklist"][:na])
        assert np.array_equal(da["particleindices"][:nass], db["particleindices"][:nass])


def test_noalloc_allocates_nothing_after_warm_up(tb):
    """After one warm-up call on the device (which may load the module and so
    reserve the fixed array), further calls leave the device's free memory
    unchanged: nothing is allocated, by the library or by the driver."""
    rng = np.random.default_rng(7)
    mesh = tb.CartesianMesh(1 / 64, (0.0, 1.0), (0.0, 1.0), (0.0, 1.0))
    n = 200_000
    P = tb.Particles(n, 3, np.float32)
    P.x[...] = rng.uniform(0.0, 1.0, size=(3, n)).astype(np.float32)
    Pd = P.to("torch", device="cuda")
    part = tb.Partition(mesh, n, backend="torch", device="cuda")
    lib = tb._abi.load_library()
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    args = (C.byref(mesh.struct()), C.byref(Pd.struct()), 1, C.byref(part.struct()), C.c_void_p(stream),
            None, None, err, 256)
    assert lib.tb_bin_particles_noalloc(*args) == tb._abi.TB_OK, err.value.decode()  # warm-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert lib.tb_bin_particles_noalloc(*args) == tb._abi.TB_OK, err.value.decode()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_oversized_input(tb):
    lib = tb._abi.load_library()
    mesh = tb.CartesianMesh(1 / 64, (0.0, 1.0), (0.0, 1.0), (0.0, 1.0))
    P = tb.Particles(0, 3, np.float32)
    s = P.struct()
    s.n = (1 << 20) + 1  # rejected before any pointer is read
    part = tb.Partition(mesh, 0)
    err = C.create_string_buffer(256)
    rc = lib.tb_bin_particles_noalloc(C.byref(mesh.struct()), C.byref(s), 1, C.byref(part.struct()), None,
                                      None, None, err, 256)
    assert rc == tb._abi.TB_ERR_CAPACITY
    assert b"fixed scratch limit" in err.value
