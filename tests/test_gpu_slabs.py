"""The z-slab decomposition on the device: two ranks of tesserae_b200.slabs
with DeviceBackend (libtesserae_b200's binning, P2G, grid half and G2P on
device state, FP64), run as two host threads on one GPU with an in-process
stand-in for torch.distributed's send / recv (each rank its own library
context and CUDA stream; no kernel waits on the other rank, the ranks only
wait on the host for each other's messages), against the one-rank oracle
rollout, every particle found by its global id (1e-12 relative)."""
import queue
import threading

import numpy as np
import pytest

from slab_scene import scene

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
NSTEPS = 6


class LoopbackDist:
    """send / recv between threads of one process: isend enqueues a copy,
    irecv's wait() dequeues into the given tensor (same order per peer pair)."""

    def __init__(self, rank, boxes):
        self.rank, self.boxes = rank, boxes

    class _Req:
        def __init__(self, fn=None):
            self.fn = fn

        def wait(self):
            if self.fn:
                self.fn()

    def isend(self, t, peer):
        self.boxes[(self.rank, peer)].put(t.clone())
        return self._Req()

    def irecv(self, t, peer):
        def fn():
            got = self.boxes[(peer, self.rank)].get(timeout=120)
            t.copy_(got)
        return self._Req(fn)


@pytest.mark.parametrize("walls", ["0", "1"])
def test_two_device_slabs_match_one_rank(tb, oracle, walls):
    from tesserae_b200 import runtime, slabs
    sc = scene(tb, walls == "1")
    world = 2
    boxes = {(a, b): queue.Queue() for a in range(world) for b in range(world) if a != b}
    results, errors = {}, []

    def run(rank):
        try:
            stream = torch.cuda.Stream()
            with torch.cuda.stream(stream):
                ctx = runtime.Context(0, stream=stream)
                layout = slabs.SlabLayout(sc.mesh, world, rank)
                P, ids = slabs.scatter(layout, sc.particles)
                P = P.to("torch", device="cuda")
                G = tb.generate_grid(layout.local, np.float64, backend="torch", device="cuda")
                P, ids = slabs.step(layout, slabs.DeviceBackend(ctx), P, ids, G, sc.params,
                                    LoopbackDist(rank, boxes), NSTEPS)
                ctx.synchronize()
                results[rank] = (P.numpy(), np.asarray(ids.cpu() if hasattr(ids, "cpu") else ids))
                ctx.close()
        except Exception as e:  # reported by the main thread
            errors.append(repr(e))

    threads = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    ref = sc.particles.to("numpy")
    oracle.step(sc.mesh, ref, tb.generate_grid(sc.mesh), sc.params, NSTEPS)
    ids = np.concatenate([results[r][1] for r in range(world)])
    assert np.array_equal(np.sort(ids), np.arange(ref.n))
    for k in ("x", "v", "F", "sigma", "V"):
        got = np.concatenate([results[r][0][k] for r in range(world)], axis=-1)
        want = getattr(ref, k)[..., ids]
        err = np.max(np.abs(got - want)) / np.max(np.abs(want))
        assert err <= 1e-12, (k, err)
