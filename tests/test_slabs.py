"""The z-slab decomposition (tesserae_b200/slabs.py) with 2 and 3 gloo ranks on
CPU against the one-rank oracle rollout: every particle, found by its global
id, ends where the undecomposed step puts it (x, v, F, sigma, V to 1e-12
relative; the decomposed P2G adds the same terms in another order), particles
migrated between slabs, and the slab bounds are block-aligned and cover the
domain."""
import json
import pathlib
import socket
import subprocess
import sys

import numpy as np
import pytest

from slab_scene import scene

ROOT = pathlib.Path(__file__).resolve().parent.parent
NSTEPS = 6


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,walls", [(2, "0"), (3, "1")])
def test_slabs_match_one_rank(tb, oracle, tmp_path, world, walls):
    pytest.importorskip("torch")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(world),
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           str(ROOT / "tests" / "slab_worker.py"), str(tmp_path), walls, str(NSTEPS)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    sc = scene(tb, walls == "1")
    ref = sc.particles.to("numpy")
    oracle.step(sc.mesh, ref, tb.generate_grid(sc.mesh), sc.params, NSTEPS)
    metas = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in range(world)]
    # block-aligned slabs that tile the domain
    assert metas[0]["c0"] == 0 and metas[-1]["c1"] == sc.mesh.n_nodes[2] - 1
    assert all(a["c1"] == b["c0"] and a["c1"] % 4 == 0 for a, b in zip(metas, metas[1:]))
    parts = [np.load(tmp_path / f"rank{k}.npz") for k in range(world)]
    ids = np.concatenate([p["ids"] for p in parts])
    assert np.array_equal(np.sort(ids), np.arange(ref.n))  # every particle exactly once
    assert any(m["n_end"] != m["n_start"] for m in metas)  # particles migrated
    for k in ("x", "v", "F", "sigma", "V"):
        got = np.concatenate([p[k] for p in parts], axis=-1)
        want = getattr(ref, k)[..., ids]
        err = np.max(np.abs(got - want)) / np.max(np.abs(want))
        assert err <= 1e-12, (k, err)
