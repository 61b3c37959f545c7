"""One rank of the z-slab check (launched by tests/test_slabs.py with
torch.distributed.run, gloo, on CPU): the rank takes its slab of a seeded scene
whose particles cross slab faces, advances it with tesserae_b200.slabs.step
(P2G, the shared-layer sum-exchange, grid half, G2P, migration), the phases
computed by the CPU oracle, and writes its particles with their global ids."""
import json
import os
import pathlib
import sys

import numpy as np
import torch.distributed as dist

sys.path.insert(0, str(pathlib.Path(__file__).resolve().parent))
import conftest  # noqa: E402
from slab_scene import scene  # noqa: E402


class OracleBackend:
    def __init__(self, oracle):
        self.o = oracle

    def p2g(self, mesh, P, grid, params):
        self.o.p2g(mesh, P, grid, params)

    def grid_update(self, mesh, grid, params):
        self.o.grid_update(mesh, grid, params)

    def g2p(self, mesh, grid, P, params):
        self.o.g2p(mesh, grid, P, params)


def main(out_dir: str, walls: str, nsteps: str):
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo")
    tb = conftest.load_package()
    from tesserae_b200 import slabs
    oracle = conftest.load_oracle_module().Oracle(tb._abi)
    sc = scene(tb, walls == "1")
    layout = slabs.SlabLayout(sc.mesh, world, rank)
    P, ids = slabs.scatter(layout, sc.particles)
    G = tb.generate_grid(layout.local)
    n0 = P.n
    P, ids = slabs.step(layout, OracleBackend(oracle), P, ids, G, sc.params, dist, int(nsteps))
    np.savez(pathlib.Path(out_dir, f"rank{rank}.npz"), ids=ids, **{k: v for k, v in P.numpy().items()})
    pathlib.Path(out_dir, f"rank{rank}.json").write_text(json.dumps(
        {"rank": rank, "c0": layout.c0, "c1": layout.c1, "n_start": n0, "n_end": P.n}))
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main(*sys.argv[1:4])
