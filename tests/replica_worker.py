"""One rank of the replica-path check (launched by tests/test_replicas.py with
torch.distributed.run, gloo, on CPU): each rank builds the same block-ordered
scene, advances its own replica with the CPU oracle, and reduces its time with
bench.py's helpers exactly as bench.py does on the GPU ranks."""
import hashlib
import importlib.util
import json
import os
import pathlib
import sys
import time

import numpy as np
import torch.distributed as dist

ROOT = pathlib.Path(__file__).resolve().parent.parent


def main(out_dir: str):
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo")
    spec = importlib.util.spec_from_file_location("bench", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    tb = bench.load_package()
    oracle = bench.load_oracle(tb).Oracle(tb._abi)
    sc = tb.scenes.block_ordered(tb.scenes.cube3d(scale=32))
    digest = hashlib.sha256(np.ascontiguousarray(sc.particles.x).tobytes()).hexdigest()
    G = tb.generate_grid(sc.mesh)
    steps = 2
    t0 = time.perf_counter()
    oracle.step_parallel(sc.mesh, sc.particles, G, sc.params, steps, 1)
    if rank == 1:
        time.sleep(0.3)  # the slower replica sets the job time
    local_ms = 1e3 * (time.perf_counter() - t0)
    ms = bench.max_over_ranks(local_ms, dist, "cpu")
    value = bench.job_throughput(world, sc.particles.n, steps, ms)
    x_sum = float(np.sum(sc.particles.x))
    pathlib.Path(out_dir, f"rank{rank}.json").write_text(json.dumps(
        {"rank": rank, "world": world, "digest": digest, "local_ms": local_ms, "ms": ms, "value": value,
         "n": sc.particles.n, "steps": steps, "x_sum": x_sum}))
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main(sys.argv[1])
