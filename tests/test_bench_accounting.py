"""bench.py's roofline accounting: the algorithmic bytes per particle-step and
per active node of the three forms (FP64: 504 B and 208 B; FP32 state with FP64
F: 328 B and 104 B; the same with FP64 positions: 376 B and 104 B), the per-kernel
figures they are built from, the ncu traffic file it scales, and the whole-job
throughput of N replicas."""
import importlib.util
import pathlib

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("s,sx,per_p,per_n", [(8, 8, 504, 208), (4, 4, 328, 104), (4, 8, 376, 104)])
def test_step_bytes(bench, s, sx, per_p, per_n):
    assert bench.step_bytes(s, sx) == (per_p, per_n)


def test_kernel_bytes_add_up(bench):
    for s, sx in ((8, 8), (4, 4), (4, 8)):
        p2g, g2p = bench.algorithmic_bytes("p2g", s, sx), bench.algorithmic_bytes("g2p", s, sx)
        binning = 3 * sx + 8  # x read; block id and particle index written
        assert bench.step_bytes(s, sx)[0] == binning + p2g[0] + g2p[0]
        # per active node: P2G writes m, mv, f; the grid update reads them and
        # writes v, vn; G2P reads v, vn
        assert bench.step_bytes(s, sx)[1] == p2g[1] + 7 * s + 6 * s + g2p[1]


def test_traffic_file_scales_by_particles(bench):
    lines = (ROOT / "profiles" / "traffic_cube3d.txt").read_text().splitlines()
    per = {k: float(v) for k, v in (l.split() for l in lines if l and not l.startswith("#"))}
    assert set(per) >= {"p2g", "g2p"}
    n = 16_777_216
    assert bench.read_traffic("p2g", n) == pytest.approx(per["p2g"] * n)
    assert bench.read_traffic("nonexistent", n) is None


def test_job_throughput(bench):
    assert bench.job_throughput(1, 1000, 10, 2.0) == pytest.approx(5e6)
    assert bench.job_throughput(4, 1000, 10, 2.0) == pytest.approx(2e7)
    assert bench.max_over_ranks(3.5) == 3.5  # one rank: its own time


@pytest.mark.parametrize("s,sx", [(8, 8), (4, 4), (4, 8)])
def test_config_bytes(bench, s, sx):
    # the plain equation set is the headline's accounting
    assert bench.config_bytes(s, sx) == bench.step_bytes(s, sx)
    # per-particle mass (P2G) and Lame parameters (G2P) are one scalar read each
    assert bench.config_bytes(s, sx, ("m",))[0] == bench.step_bytes(s, sx)[0] + s
    assert bench.config_bytes(s, sx, ("mu", "lam"))[0] == bench.step_bytes(s, sx)[0] + 2 * s
    # APIC: B read in P2G and written in G2P, the old velocity and vn not read
    pp, pn = bench.config_bytes(s, sx, apic=True)
    assert pp == bench.step_bytes(s, sx)[0] + 18 * s - 3 * s
    assert pn == bench.step_bytes(s, sx)[1] - 3 * s


def test_fd_summary_normalises_by_field_rms(bench):
    """fd_summary: per form the largest per-direction relative error and the
    largest error over the field's RMS derivative."""
    checks = [{"field": "v", "fd": 1.0, "adjoint_f64": 1.0, "adjoint_x64": 1.0001, "adjoint_f32": 1.001},
              {"field": "v", "fd": 0.01, "adjoint_f64": 0.01, "adjoint_x64": 0.0101, "adjoint_f32": 0.011}]
    for ch in checks:
        for f in ("f64", "x64", "f32"):
            ch[f"rel_err_{f}"] = abs(ch[f"adjoint_{f}"] - ch["fd"]) / abs(ch["fd"])
    out = bench.fd_summary(checks, 2)
    rms = ((1.0 + 1e-4) / 2) ** 0.5
    assert abs(out["max_rel_err_x64"] - 0.01) < 1e-12
    assert abs(out["max_err_over_rms_x64"] - 1e-4 / rms) < 1e-12
    assert out["max_rel_err_fp32_tape"] == out["max_rel_err_x64"]
