"""The multi-GPU path is replicas only (no data-path collective): bench.py runs
the same workload on every rank and reports the whole-job throughput from the
slowest rank's time. Checked here with two gloo ranks on CPU through
torch.distributed.run, as the GPU bench is launched: every rank builds the same
scene, both ranks agree on the job time, which is the max of their own times,
and the throughput counts both replicas."""
import json
import pathlib
import socket
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_replicas_gloo(tmp_path):
    pytest.importorskip("torch")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           str(ROOT / "tests" / "replica_worker.py"), str(tmp_path)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    res = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in range(2)]
    assert res[0]["digest"] == res[1]["digest"]  # the same replica on every rank
    assert res[0]["x_sum"] == res[1]["x_sum"]    # and the same result after its steps
    assert res[0]["ms"] == res[1]["ms"] == max(res[0]["local_ms"], res[1]["local_ms"])
    assert res[1]["local_ms"] > res[0]["local_ms"]
    n, steps = res[0]["n"], res[0]["steps"]
    assert res[0]["value"] == pytest.approx(2 * n * steps / (res[0]["ms"] * 1e-3), rel=1e-12)
