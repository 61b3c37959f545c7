"""Benchmark of the explicit MPM step (bin -> P2G -> grid update -> G2P).

Workload: the 3D cube scene (unit cube 256^3 cells, centre cube of side 0.5 at
2^3 particles per cell = 16 777 216 particles, Neo-Hookean E = 1e6, nu = 0.3,
gravity), seeded synthetic data. One bench "step" = one MPM step over all
particles. The headline form is the mixed FP32 step with FP64 positions (FP32
velocity, stress, volume, weights and transfers; FP64 x, F, det F, log J; P2G
partials summed in FP64), the form that holds the 100-step error against the
FP64 run below 1e-5. The same step with FP32 positions and the plain FP64 step
are measured beside it, with their accuracy.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0). N > 1 (torchrun): every rank runs its own
replica of the workload (weak scaling, no data exchange); time = max over ranks.
`--impl reference` times the reference's CPU algorithm (the OpenMP restatement
in oracle/, FP64, all host cores) on the same workload.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import pathlib
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
METRIC = "particle-steps/s, 1 B200: FP32 fused vs FP64 plain @<=1e-5 rel err; adj/fwd"


def load_package():
    if "tesserae_b200" in sys.modules:
        return sys.modules["tesserae_b200"]
    pkg = ROOT / "tesserae.jl_b200"
    spec = importlib.util.spec_from_file_location("tesserae_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["tesserae_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle(tb):
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as oracle_mod  # noqa: E402  (CPU baseline / reference arm only)
    return oracle_mod


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled through NVML every
    10 ms from a background thread while the timed region runs; nvidia-smi is
    the fallback when NVML cannot be loaded."""

    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                   "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.sm, self.smax, self.reasons, self.source = [], None, set(), None
        self._stop = None
        self._thread = None
        self._proc = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        # the CUDA ordinal and the NVML index differ under CUDA_VISIBLE_DEVICES: match by UUID
        try:
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            for cand in (uuid, "GPU-" + uuid):
                try:
                    return pynvml, pynvml.nvmlDeviceGetHandleByUUID(cand)
                except Exception:
                    pass
        except Exception:
            pass
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def _sample(self, nv, h):
        self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
        get = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        bits = int(get(h))
        for name, bit in self.REASON_BITS.items():
            if bits & bit:
                self.reasons.add(name)

    def __enter__(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._stop = threading.Event()

            def run():
                while not self._stop.is_set():
                    try:
                        self._sample(nv, h)
                    except Exception:
                        pass
                    self._stop.wait(0.01)

            self._nv, self._h = nv, h
            self._thread = threading.Thread(target=run, daemon=True)
            self._thread.start()
            self.source = "nvml"
        except Exception:
            try:
                self._proc = subprocess.Popen(
                    ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                     "--format=csv,noheader,nounits", "-lms", "100"],
                    stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.source = "nvidia-smi"
            except OSError:
                self._proc = None
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            if not self.sm:  # a region shorter than one period: take one sample now
                try:
                    self._sample(self._nv, self._h)
                except Exception:
                    pass
            self._stop.set()
            self._thread.join(timeout=5)
        if self._proc is not None:
            self._proc.terminate()
            try:
                out, _ = self._proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
                out, _ = self._proc.communicate()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for l in out.splitlines():
                f = [x.strip() for x in l.split(",")]
                if len(f) < 9:
                    continue
                try:
                    self.sm.append(float(f[1]))
                    self.smax = float(f[2])
                except ValueError:
                    continue
                for name, val in zip(names, f[5:9]):
                    if val.lower().startswith("active"):
                        self.reasons.add(name)

    def summary(self) -> dict:
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.smax,
                "reasons": sorted(self.reasons), "samples": len(self.sm), "source": self.source}


def max_over_ranks(v: float, dist=None, device: str = "cuda") -> float:
    """The max of a per-rank time over all ranks (every rank gets it): the
    job-level time of N replicas. `dist` is torch.distributed or None (one rank)."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world: int, n: int, steps: int, ms: float) -> float:
    """Whole-job particle-steps/s of `world` replicas of an n-particle workload
    that each ran `steps` steps, the slowest in `ms` milliseconds."""
    return world * n * steps / (ms * 1e-3)


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Algorithmic bytes per particle and per active node of each kernel family:
# the scatter/gather reads and writes of the reference's equations (weights
# evaluated in the kernels), for a state scalar of `s` bytes and positions of
# `sx` bytes (FP64 positions in the headline form); F is FP64 in every form.
def algorithmic_bytes(kind: str, s: int, sx: int) -> tuple[int, int]:
    per_p = {
        # x, v, V, sigma(6) read
        "p2g": 3 * sx + (3 + 1 + 6) * s,
        # x, v, F(9 x 8) read; x, v, grad_v(9), F, sigma(6), V written
        "g2p": 3 * sx + 3 * s + 72 + 3 * sx + (3 + 9 + 6 + 1) * s + 72,
        # x read, block id written
        "bin_count": 3 * sx + 4,
    }[kind]
    per_n = {
        "p2g": 7 * s,       # m, mv, f written once per active node
        "g2p": 6 * s,       # v, vn read once per active node
        "bin_count": 0,
    }[kind]
    return per_p, per_n


def step_bytes(s: int, sx: int) -> tuple[int, int]:
    """Algorithmic bytes of one whole MPM step per particle and per active node:
    binning (x read; block id and particle index written), P2G, G2P; per active
    node the P2G result write, the grid update's read and write and the G2P read."""
    per_p = (3 * sx + 8) + algorithmic_bytes("p2g", s, sx)[0] + algorithmic_bytes("g2p", s, sx)[0]
    per_n = 7 * s + 7 * s + 6 * s + 6 * s
    return per_p, per_n


def config_bytes(s: int, sx: int, per_particle=(), apic: bool = False) -> tuple[int, int]:
    """Algorithmic bytes of one whole step per particle and per active node for
    a config: state scalars of `s` bytes, positions of `sx`, F FP64.
    `per_particle` names the optional per-particle inputs (m and l read by P2G,
    mu, lam and V0 by G2P). APIC reads B in P2G and writes it in G2P, and its
    G2P reads neither the particle's old velocity nor the nodes' vn."""
    p2g = 3 * sx + (3 + 1 + 6) * s + (9 * s if apic else 0) + s * sum(k in per_particle for k in ("m", "l"))
    g2p_read = 3 * sx + (0 if apic else 3 * s) + 72 + s * sum(k in per_particle for k in ("mu", "lam", "V0", "l"))
    g2p_write = 3 * sx + (3 + 9 + 6 + 1) * s + 72 + (9 * s if apic else 0)
    per_p = (3 * sx + 8) + p2g + g2p_read + g2p_write
    per_n = 7 * s + 7 * s + 6 * s + (3 * s if apic else 6 * s)
    return per_p, per_n


FORMS = {
    # name: (state dtype, FP64 positions, description)
    "x64": (np.float32, True, "mixed FP32 with FP64 positions (FP64 x, F, det F, log J; FP64-summed P2G partials)"),
    "f32": (np.float32, False, "mixed FP32 with FP32 positions (FP64 F, det F, log J; FP64-summed P2G partials)"),
    "f64": (np.float64, False, "plain FP64"),
}


def read_traffic(kernel: str, n: int):
    """DRAM bytes (read + write) per launch of `kernel` on the full workload,
    scaled from the committed ncu capture's per-particle figure
    (profiles/traffic_cube3d.txt: lines `<kernel> <bytes per particle>`)."""
    f = ROOT / "profiles" / "traffic_cube3d.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        parts = line.split()
        if len(parts) == 2 and parts[0] == kernel:
            return float(parts[1]) * n
    return None


def active_nodes(mesh, particles_np) -> int:
    """Nodes inside the support of at least one particle (quadratic B-spline)."""
    x = particles_np
    n = mesh.n_nodes
    lo = [np.floor((x[d] - mesh.xmin[d]) * mesh.h_inv - 0.5).astype(np.int64) for d in range(3)]
    mask = np.zeros(n[::-1], dtype=bool)  # z, y, x
    mins = [int(l.min()) for l in lo]
    maxs = [int(l.max()) + 2 for l in lo]
    # the cube scene fills a box of cells densely: the active nodes are that box
    for d in range(3):
        mins[d], maxs[d] = max(mins[d], 0), min(maxs[d], n[d] - 1)
    mask[mins[2]:maxs[2] + 1, mins[1]:maxs[1] + 1, mins[0]:maxs[0] + 1] = True
    return int(mask.sum())


# The reference's published GPU numbers for the Taylor impact on an RTX 5090
# (docs/src/gpu.md:215-220: 31 s FP64, 8 s FP32), as particle-steps/s with the
# tutorial's 1 472 942 particles and 1 833 steps (taylor_impact.jl:84, 265-267).
TAYLOR_PUBLISHED = {"fp64": 1472942 * 1833 / 31.0, "fp32": 1472942 * 1833 / 8.0}


def taylor_leg(tb, runtime, ctx, steps: int = 200, warmup: int = 5, cpu_steps: int = 2) -> dict:
    """The Taylor impact of docs/src/gpu.md:202-392 at full size (1.48 M
    particles, KernelCorrection(BSpline(Quadratic())), von Mises, slip floor):
    `steps` steps of its adaptive loop (each takes dt = 0.8 h / max c from a
    device reduction read back on the host, as the reference's
    `maximum(particles.c)`, then runs one step) after `warmup` steps, timed
    between CUDA events, in each precision form; against the reference's
    published RTX 5090 throughput of the same loop. Also the oracle port's FP64
    step on the host cores over `cpu_steps` steps."""
    import torch
    sc = tb.scenes.taylor3d()
    mesh, prm, host = sc.mesh, sc.params, sc.particles
    n = host.n
    out = {"workload": f"Taylor impact (docs/src/gpu.md:202-392): {n} particles, mesh "
                       f"{'x'.join(str(k) for k in mesh.n_nodes)} nodes (h = R/12), KernelCorrection(BSpline(Quadratic())), "
                       "von Mises (H = 0.1 GPa, tau_y0 = 0.4 GPa), 227 m/s onto a slip floor, dt = 0.8 h / max c per step",
           "n_particles": n, "steps": steps, "warmup": warmup, "unit": "particle-steps/s",
           "published_rtx5090": TAYLOR_PUBLISHED,
           "note": "each step includes its wave-speed reduction and the host read of max c"}
    for name, dtype, x64 in (("fp64", np.float64, False), ("fp32", np.float32, False),
                             ("fp32_x64", np.float32, True)):
        P = host.to("torch", device="cuda", dtype=dtype, x64=x64)
        part = tb.Partition(mesh, n, backend="torch", device="cuda")
        G = tb.generate_grid(mesh, dtype, backend="torch", device="cuda")
        runtime.adaptive_steps(G, P, part, mesh, prm, warmup, ctx=ctx)
        ctx.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        t_sim = runtime.adaptive_steps(G, P, part, mesh, prm, steps, ctx=ctx)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        d = P.numpy()
        out[name] = {"value": n * steps / (ms * 1e-3), "ms_per_step": ms / steps,
                     "simulated_us": (t_sim * 1e6), "plastic_particles": int(np.sum(d["eps_p"] > 0)),
                     "max_eps_p": float(np.max(d["eps_p"])), "finite": bool(np.isfinite(d["x"]).all()),
                     "full_run_s_1805_steps": 1805 * ms * 1e-3 / steps}
        ref = TAYLOR_PUBLISHED["fp64" if name == "fp64" else "fp32"]
        out[name]["over_published_rtx5090"] = out[name]["value"] / ref
        del P, part, G
        torch.cuda.empty_cache()
    if cpu_steps > 0:
        orc = load_oracle(tb).Oracle(tb._abi)
        Pc = host.to("numpy")
        Gc = tb.generate_grid(mesh)
        prm1 = type(prm).from_buffer_copy(prm)
        orc.step_parallel(mesh, Pc, Gc, prm1, 1)
        t0 = time.perf_counter()
        orc.step_parallel(mesh, Pc, Gc, prm1, cpu_steps)
        cs = time.perf_counter() - t0
        out["cpu_port"] = {"value": n * cpu_steps / cs, "cores": orc.max_threads(),
                           "sample": f"{cpu_steps} FP64 steps after 1 warm-up, OpenMP colour-phased restatement"}
    return out


def adjoint_leg(tb, runtime, ctx, scale: int = 1, every: int = 20, fd_directions: int = 32) -> dict:
    """Differentiable rollout on the sphere scene (64^3 cells, ~1.9M particles,
    200 steps), mixed FP32 form with FP64 positions (the headline form): device
    time of the plain forward rollout, the taped forward and the backward
    pass for the centre-of-mass loss, with the whole tape held in HBM (every
    step's state, grid and partition: the backward pass runs the adjoint kernels
    only) and with checkpoints every `every` steps (the backward pass re-runs
    each segment); plus directional derivatives of a linear loss on the final
    positions along `fd_directions` random directions per field, from the FP64
    tape, the mixed form's tape and the mixed form with FP32 positions, against
    central differences of the FP64 device rollout."""
    import torch
    sc = tb.scenes.sphere3d(scale=scale)
    mesh, prm, host = sc.mesh, sc.params, sc.particles
    n, nsteps = host.n, sc.nsteps
    part = tb.Partition(mesh, n, backend="torch", device="cuda")
    G32 = tb.generate_grid(mesh, np.float32, backend="torch", device="cuda")

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    P = host.to("torch", device="cuda", dtype=np.float32, x64=True)
    runtime.step(G32, P, part, mesh, prm, 3, ctx=ctx)  # warm-up
    P = host.to("torch", device="cuda", dtype=np.float32, x64=True)
    fwd_ms = timed(lambda: runtime.step(G32, P, part, mesh, prm, nsteps, ctx=ctx))
    c = torch.tensor(sc.meta["target"], dtype=torch.float64, device="cuda")[:, None]

    def tape_run(k):
        # warm-up of the tape: its buffers are allocated once per context
        # (grow-only) on the first call, outside the timed region
        Q = host.to("torch", device="cuda", dtype=np.float32, x64=True)
        runtime.tape_forward(G32, Q, part, mesh, prm, nsteps, k, ctx=ctx)
        adj_w = tb.Adjoint(n, 3, backend="torch", device="cuda")
        runtime.tape_backward(G32, Q, part, mesh, prm, adj_w, ctx=ctx)
        del adj_w, Q
        Q = host.to("torch", device="cuda", dtype=np.float32, x64=True)
        tape_ms = timed(lambda: runtime.tape_forward(G32, Q, part, mesh, prm, nsteps, k, ctx=ctx))
        r = Q.x.double().mean(dim=1, keepdim=True) - c
        loss = float((r ** 2).sum())
        adj = tb.Adjoint(n, 3, backend="torch", device="cuda")
        adj.x.copy_((2 * r / n).expand(-1, n))
        bwd_ms = timed(lambda: runtime.tape_backward(G32, Q, part, mesh, prm, adj, ctx=ctx))
        return Q, adj, loss, tape_ms, bwd_ms

    # the whole tape first (timed), then the checkpointed one, whose backward is
    # also split per kernel
    P, adj, loss, tape_ms, bwd_ms = tape_run(1)
    glogE = adj.mu * P.mu.double() + adj.lam * P.lam.double()
    gnorm_v, gnorm_logE = float(adj.v.norm()), float(glogE.norm())
    ctx.profile(True)
    runtime.tape_backward(G32, P, part, mesh, prm, adj, ctx=ctx)
    kt_full = ctx.profile_read()
    ctx.profile(False)
    ctx.release_tape()
    del adj
    P, adj, _, tape_ck_ms, bwd_ck_ms = tape_run(every)
    ctx.profile(True)
    runtime.tape_forward(G32, P, part, mesh, prm, every, every, ctx=ctx)
    ctx.profile_read()
    runtime.tape_backward(G32, P, part, mesh, prm, adj, ctx=ctx)
    kt = ctx.profile_read()
    ctx.profile(False)
    del adj

    # finite-difference check: L = sum c . x_T with random c, gradients from the
    # FP64 tape (the check of the adjoint itself) and from the FP32 tape
    rng = np.random.default_rng(17)
    cw = rng.normal(size=(3, n))
    G64 = tb.generate_grid(mesh, np.float64, backend="torch", device="cuda")

    def grads(dtype, G, x64=False):
        Q = host.to("torch", device="cuda", dtype=dtype, x64=x64)
        runtime.tape_forward(G, Q, part, mesh, prm, nsteps, every, ctx=ctx)
        adj_c = tb.Adjoint(n, 3, backend="torch", device="cuda")
        adj_c.x.copy_(torch.from_numpy(cw))
        runtime.tape_backward(G, Q, part, mesh, prm, adj_c, ctx=ctx)
        return adj_c.numpy()

    gs = {"f64": grads(np.float64, G64), "x64": grads(np.float32, G32, x64=True), "f32": grads(np.float32, G32)}
    ctx.release_tape()

    def loss64(Q):
        Qd = Q.to("torch", device="cuda")
        runtime.step(G64, Qd, part, mesh, prm, nsteps, ctx=ctx)
        ctx.synchronize()
        return float(np.sum(cw * Qd.x.cpu().numpy()))

    checks = []
    for k in range(fd_directions):
        for field, eps in (("v", 1e-5), ("logE", 1e-4)):
            d = rng.normal(size=(3, n) if field == "v" else (n,))
            Qp, Qm = host.to("numpy"), host.to("numpy")
            if field == "v":
                Qp.v += eps * d
                Qm.v -= eps * d
                ad = {f: float(np.sum(g["v"] * d)) for f, g in gs.items()}
            else:
                Qp.mu *= np.exp(eps * d)
                Qp.lam *= np.exp(eps * d)
                Qm.mu *= np.exp(-eps * d)
                Qm.lam *= np.exp(-eps * d)
                ad = {f: float(np.sum((g["mu"] * host.mu + g["lam"] * host.lam) * d)) for f, g in gs.items()}
            fd = (loss64(Qp) - loss64(Qm)) / (2 * eps)
            checks.append({"field": field, "fd": fd, **{f"adjoint_{f}": a for f, a in ad.items()},
                           **{f"rel_err_{f}": abs(a - fd) / max(abs(fd), 1e-30) for f, a in ad.items()}})
    del G64, P
    torch.cuda.empty_cache()
    adj_ms = sum(v[1] for k, v in kt.items() if k.startswith("adj_")) / every
    return {
        "value": (tape_ms + bwd_ms) / fwd_ms,
        "backward_over_forward": bwd_ms / fwd_ms,
        "workload": f"sphere3d: 64^3 cells, sphere r=0.3, {n} particles, {nsteps} steps, whole tape in HBM "
                    f"(checkpointed every {every} beside it), mixed FP32 form with FP64 positions; "
                    f"loss = |x_com - (0.5, 0.5, 0.8)|^2",
        "n_particles": n, "steps": nsteps, "loss": loss,
        "forward_ms_per_step": fwd_ms / nsteps, "tape_forward_ms_per_step": tape_ms / nsteps,
        "backward_ms_per_step": bwd_ms / nsteps,
        "tape_bytes_per_step": runtime.tape_slot_bytes(mesh, n, np.float32, x64=True),
        "grad_v0_norm": gnorm_v, "grad_logE_norm": gnorm_logE,
        "backward_kernels_ms_per_step": {k: v[1] / nsteps for k, v in sorted(kt_full.items())},
        "checkpointed": {
            "checkpoint_every": every,
            "value": (tape_ck_ms + bwd_ck_ms) / fwd_ms,
            "backward_over_forward": bwd_ck_ms / fwd_ms,
            "tape_forward_ms_per_step": tape_ck_ms / nsteps, "backward_ms_per_step": bwd_ck_ms / nsteps,
            # the backward step's two parts: the forward recomputed from the last
            # checkpoint (binning, P2G, grid, G2P kernels) and the adjoint kernels
            "backward_split": {
                "recompute_ms_per_step": sum(v[1] for k, v in kt.items() if not k.startswith("adj_")) / every,
                "adjoint_kernels_ms_per_step": adj_ms,
                "adjoint_kernels_over_forward": adj_ms / (fwd_ms / nsteps)}},
        "fd_check": fd_summary(checks, fd_directions),
    }


def fd_summary(checks, fd_directions) -> dict:
    """Finite-difference check summary: per tape form the largest error relative
    to each direction's own derivative, and relative to the RMS derivative of
    its field (a direction whose derivative nearly cancels has a large
    relative error from the same absolute error)."""
    out = {"against": "central differences of the FP64 device rollout, L = sum c . x_T, random c",
           "directions_per_field": fd_directions,
           "forms": {"f64": "FP64 tape", "x64": "mixed FP32 tape with FP64 positions (the headline form)",
                     "f32": "mixed FP32 tape with FP32 positions"}}
    rms = {}
    for ch in checks:
        rms.setdefault(ch["field"], []).append(ch["fd"] ** 2)
    rms = {f: float(np.sqrt(np.mean(v))) for f, v in rms.items()}
    for form in ("f64", "x64", "f32"):
        out[f"max_rel_err_{form}"] = max(ch[f"rel_err_{form}"] for ch in checks)
        out[f"max_err_over_rms_{form}"] = max(abs(ch[f"adjoint_{form}"] - ch["fd"]) / rms[ch["field"]]
                                              for ch in checks)
    out["max_rel_err"] = out["max_rel_err_f64"]
    out["max_rel_err_fp32_tape"] = out["max_rel_err_x64"]
    out["directions"] = checks
    return out


def _form_particles(tb, runtime, ctx, sc, name, device="cuda"):
    """Device particles of scene `sc` in precision form `name` (x64 / f32 / f64),
    stored in block order: binned once and put through reorder_particles!
    (threshold 1: always), the set-up docs/src/parallel.md:47-57 gives a GPU run."""
    dtype, x64, _ = FORMS[name]
    if sc.meta.get("built_on_device"):
        P = tb.scenes.dambreak3d(scale=sc.meta["scale"], device=device, dtype=dtype, x64=x64).particles
    else:
        P = sc.particles.to("torch", device=device, dtype=dtype, x64=x64)
    part = tb.Partition(sc.mesh, P.n, backend="torch", device=device)
    runtime.update(part, P, sc.mesh, ctx=ctx)
    runtime.reorder_particles(P, part, 1.0, ctx=ctx)
    del part
    return P


def config_leg(tb, runtime, ctx, sc, forms, steps: int, warmup: int, acc_steps: int, peak: float,
               per_particle=(), apic=False, sparse_forms=()) -> dict:
    """One configuration: device time per step of each precision form (a fused
    call of `steps` steps after `warmup`), its per-kernel split, the whole-step
    and dominant-kernel roofline fractions, and the FP32 form's error against
    the FP64 form after `acc_steps` steps from the same initial state. For each
    form in `sparse_forms`, the same timing on a block-sparse grid (SpGrid,
    its sparsity updated every step), its grid memory against the dense grid's,
    and its state after `steps` steps against the dense grid's."""
    import torch
    mesh, prm = sc.mesh, sc.params
    out = {"n_particles": None, "steps": steps, "warmup": warmup, "forms": {}}
    finals = {}
    for name in forms:
        P = _form_particles(tb, runtime, ctx, sc, name)
        n = P.n
        out["n_particles"] = n
        dtype = FORMS[name][0]
        part = tb.Partition(mesh, n, backend="torch", device="cuda")
        G = tb.generate_grid(mesh, dtype, backend="torch", device="cuda")
        runtime.step(G, P, part, mesh, prm, warmup, ctx=ctx)
        ctx.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ctx.launches
        torch.cuda.synchronize()
        e0.record()
        runtime.step(G, P, part, mesh, prm, steps, ctx=ctx)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        launches = (ctx.launches - l0) / steps
        nact = int((G.m != 0).sum())
        ctx.profile(True)
        runtime.step(G, P, part, mesh, prm, 3, ctx=ctx)
        kt = ctx.profile_read()
        ctx.profile(False)
        s_b = np.dtype(dtype).itemsize
        sx = 8 if FORMS[name][1] else s_b
        bp, bn = config_bytes(s_b, sx, per_particle, apic)
        alg = n * bp + nact * bn
        kern = {k: v[1] / 3 for k, v in sorted(kt.items())}
        dom = max(kern, key=kern.get)
        out["forms"][name] = {
            "form": FORMS[name][2], "ms_per_step": ms, "value": n / (ms * 1e-3), "launches_per_step": launches,
            "active_nodes": nact, "bytes_per_particle": bp, "bytes_per_active_node": bn, "step_bytes": alg,
            "step_roofline_frac": alg / (ms * 1e-3) / 1e9 / peak, "kernels_ms_per_step": kern,
            "dominant_kernel": dom, "dominant_kernel_share": kern[dom] / sum(kern.values())}
        del part, G, P
        torch.cuda.empty_cache()
        # accuracy run from the initial state
        P = _form_particles(tb, runtime, ctx, sc, name)
        part = tb.Partition(mesh, n, backend="torch", device="cuda")
        G = tb.generate_grid(mesh, dtype, backend="torch", device="cuda")
        x0 = P.x.double().clone()
        runtime.step(G, P, part, mesh, prm, acc_steps, ctx=ctx)
        ctx.synchronize()
        finals[name] = {"x": P.x.double(), "v": P.v.double(), "x0": x0,
                        "finite": bool(torch.isfinite(P.x).all() and torch.isfinite(P.v).all())}
        del part, G, P
        torch.cuda.empty_cache()
    for name in sparse_forms:
        dtype = FORMS[name][0]
        s_b = np.dtype(dtype).itemsize
        nfield = 1 + 4 * mesh.dim
        res = {}
        for sparse in (False, True):
            P = _form_particles(tb, runtime, ctx, sc, name)
            part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
            G = tb.generate_grid(mesh, dtype, backend="torch", device="cuda", sparse=sparse)
            runtime.step(G, P, part, mesh, prm, warmup, ctx=ctx)
            ctx.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            runtime.step(G, P, part, mesh, prm, steps, ctx=ctx)
            e1.record()
            torch.cuda.synchronize()
            ctx.synchronize()
            res[sparse] = {"ms": e0.elapsed_time(e1) / steps, "x": P.x.double().clone(),
                           "nodes": G.capacity if sparse else mesh.nnodes}
            del part, G, P
            torch.cuda.empty_cache()
        dx = float(torch.linalg.vector_norm(res[True]["x"] - res[False]["x"]) /
                   torch.linalg.vector_norm(res[False]["x"]))
        out.setdefault("sparse_grid", {})[name] = {
            "ms_per_step": res[True]["ms"], "dense_ms_per_step": res[False]["ms"],
            "grid_bytes": res[True]["nodes"] * nfield * s_b, "dense_grid_bytes": mesh.nnodes * nfield * s_b,
            "rel_err_x_vs_dense": dx, "steps": warmup + steps,
            "note": "SpGrid (generate_grid(SpArray, ...)): sparsity updated on the device every step; "
                    "field arrays sized for the initial active blocks x 1.5"}
    ref = finals.get("f64")
    if ref is not None:
        def rel(a, b):
            return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
        for name, f in finals.items():
            if name == "f64":
                continue
            out["forms"][name]["accuracy"] = {
                "steps": acc_steps, "rel_err_x": rel(f["x"], ref["x"]), "rel_err_v": rel(f["v"], ref["v"]),
                "rel_err_displacement": rel(f["x"] - f["x0"], ref["x"] - ref["x0"]), "finite": f["finite"],
                "against": "plain FP64 form on the device from the same initial state"}
        fast = [k for k in forms if k != "f64"]
        if fast:
            out["fp32_over_fp64_speed"] = out["forms"]["f64"]["ms_per_step"] / out["forms"][fast[0]]["ms_per_step"]
    del finals
    torch.cuda.empty_cache()
    return out


def dambreak_adjoint_leg(tb, runtime, ctx, scale: int = 2, fd_scale: int = 4, forward: int = 80, last: int = 20,
                         every: int = 5, fd_directions: int = 2) -> dict:
    """The dam break's differentiable leg: `forward` steps, then the gradient of
    L = sum c . x at the end of `last` more steps with respect to the velocity
    field at their start (the checkpointed tape over the last steps; WLS(uGIMP)
    + APIC + fluid take the general reverse step), mixed FP32 form with FP64
    positions, at 1/scale
    of the resolution (the tape holds last/every states plus `every` steps of
    state, grid and partition: 224 GB for the full 145 M-particle scene at the
    best interval). Device times per step of the plain forward, the taped
    forward and the backward pass; the FP64 tape's directional derivatives
    against central differences of the FP64 device rollout at 1/fd_scale."""
    import torch

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def setup(sc_scale, dtype):
        sc = tb.scenes.dambreak3d(scale=sc_scale, particles=False)
        P = _form_particles(tb, runtime, ctx, tb.scenes.dambreak3d(scale=sc_scale, particles=False), "f64"
                            if dtype == np.float64 else "x64")
        part = tb.Partition(sc.mesh, P.n, backend="torch", device="cuda")
        G = tb.generate_grid(sc.mesh, dtype, backend="torch", device="cuda")
        runtime.step(G, P, part, sc.mesh, sc.params, forward, ctx=ctx)
        ctx.synchronize()
        return sc, P, part, G

    sc, P, part, G = setup(scale, np.float32)
    mesh, prm, n = sc.mesh, sc.params, P.n
    start = {k: getattr(P, k).clone() for k in P.FIELDS if getattr(P, k) is not None}

    def restore():
        for k, v in start.items():
            getattr(P, k).copy_(v)

    fwd_ms = timed(lambda: runtime.step(G, P, part, mesh, prm, last, ctx=ctx))
    restore()
    tape_ms = timed(lambda: runtime.tape_forward(G, P, part, mesh, prm, last, every, ctx=ctx))
    rng = np.random.default_rng(31)
    cw = torch.from_numpy(rng.normal(size=(3, n))).cuda()
    adj = tb.Adjoint(n, 3, backend="torch", device="cuda", lame=False, apic=True)
    adj.x.copy_(cw)
    bwd_ms = timed(lambda: runtime.tape_backward(G, P, part, mesh, prm, adj, ctx=ctx))
    ctx.profile(True)
    restore()
    runtime.tape_forward(G, P, part, mesh, prm, every, every, ctx=ctx)
    ctx.profile_read()
    a2 = tb.Adjoint(n, 3, backend="torch", device="cuda", lame=False, apic=True)
    a2.x.copy_(cw)
    runtime.tape_backward(G, P, part, mesh, prm, a2, ctx=ctx)
    kt = ctx.profile_read()
    ctx.profile(False)
    gnorm = float(adj.v.norm())
    del P, part, G, start, adj, a2
    torch.cuda.empty_cache()

    # FP64 tape against central differences of the FP64 rollout, at 1/fd_scale
    sc, P, part, G = setup(fd_scale, np.float64)
    n2 = P.n
    start = {k: getattr(P, k).clone() for k in P.FIELDS if getattr(P, k) is not None}
    cw2 = torch.from_numpy(rng.normal(size=(3, n2))).cuda()

    def restore2():
        for k, v in start.items():
            getattr(P, k).copy_(v)

    runtime.tape_forward(G, P, part, sc.mesh, sc.params, last, every, ctx=ctx)
    adj = tb.Adjoint(n2, 3, backend="torch", device="cuda", lame=False, apic=True)
    adj.x.copy_(cw2)
    runtime.tape_backward(G, P, part, sc.mesh, sc.params, adj, ctx=ctx)
    gv = adj.v.clone()
    checks = []
    for _ in range(fd_directions):
        d = torch.from_numpy(rng.normal(size=(3, n2))).cuda()
        eps = 1e-6
        Ls = []
        for sgn in (1.0, -1.0):
            restore2()
            P.v.add_(sgn * eps * d)
            runtime.step(G, P, part, sc.mesh, sc.params, last, ctx=ctx)
            ctx.synchronize()
            Ls.append(float((cw2 * P.x).sum()))
        fd = (Ls[0] - Ls[1]) / (2 * eps)
        ad = float((gv * d).sum())
        checks.append({"fd": fd, "adjoint": ad, "rel_err": abs(ad - fd) / max(abs(fd), 1e-30)})
    del P, part, G, start, adj
    torch.cuda.empty_cache()
    return {"workload": f"dambreak3d at 1/{scale} resolution ({n} particles): {forward} steps, then the gradient of "
                        f"sum c . x after {last} more steps w.r.t. the velocities at their start; tape every {every}",
            "n_particles": n, "forward_ms_per_step": fwd_ms / last, "tape_forward_ms_per_step": tape_ms / last,
            "backward_ms_per_step": bwd_ms / last, "backward_over_forward": bwd_ms / fwd_ms,
            "value": (tape_ms + bwd_ms) / fwd_ms, "grad_v_norm": gnorm,
            "backward_kernels_ms_per_step": {k: v[1] / every for k, v in sorted(kt.items())},
            "fd_check": {"scale": fd_scale, "n_particles": n2, "against": "central differences (eps 1e-6) of the "
                         "FP64 device rollout, FP64 tape", "max_rel_err": max(c["rel_err"] for c in checks),
                         "directions": checks}}


def kernel_case(tb, runtime, ctx, spec: str, steps: int, warmup: int) -> dict:
    """One scene's steps alone, the workload of the per-kernel profiler
    captures: SCENE:SCALE[:FORM][:adjoint] (FORM x64, f32 or f64; default x64).
    Without `adjoint`: `warmup` steps, then `steps` steps in one call. With it: a
    whole tape of warmup + steps steps (interval 1), then its backward pass
    (only the adjoint kernels). Prints each kernel family's device time."""
    parts = spec.split(":")
    name, scale = parts[0], int(parts[1]) if len(parts) > 1 else 1
    form = next((q for q in parts[2:] if q in FORMS), "x64")
    adjoint = "adjoint" in parts[2:]
    if name == "dambreak3d":
        sc = tb.scenes.dambreak3d(scale=scale, particles=False)
    else:
        sc = getattr(tb.scenes, name)(scale=scale)
    mesh, prm = sc.mesh, sc.params
    P = _form_particles(tb, runtime, ctx, sc, form)
    dtype = FORMS[form][0]
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(mesh, dtype, backend="torch", device="cuda")
    if adjoint:
        import torch
        runtime.tape_forward(G, P, part, mesh, prm, warmup + steps, 1, ctx=ctx)
        adj = tb.Adjoint(P.n, mesh.dim, backend="torch", device="cuda", lame=P.mu is not None,
                         apic=prm.transfer == tb._abi.TB_TRANSFER_APIC)
        gen = torch.Generator(device="cuda").manual_seed(5)
        adj.x.copy_(torch.randn(adj.x.shape, generator=gen, device="cuda", dtype=torch.float64))
        ctx.profile(True)
        runtime.tape_backward(G, P, part, mesh, prm, adj, ctx=ctx)
        kt = ctx.profile_read()
        ctx.profile(False)
        nsteps = warmup + steps
    else:
        runtime.step(G, P, part, mesh, prm, warmup, ctx=ctx)
        ctx.synchronize()
        ctx.profile(True)
        runtime.step(G, P, part, mesh, prm, steps, ctx=ctx)
        kt = ctx.profile_read()
        ctx.profile(False)
        nsteps = steps
    return {"kernel_case": spec, "n_particles": P.n, "form": form, "adjoint": adjoint, "steps": nsteps,
            "kernels_ms_per_step": {k: v[1] / nsteps for k, v in sorted(kt.items())},
            "launches_per_step": {k: v[0] / nsteps for k, v in sorted(kt.items())}}


def fullsize_oracle_check(tb, runtime, ctx, sc, nsteps: int = 3) -> dict:
    """The plain FP64 device step against the FP64 oracle (the OpenMP
    restatement of the reference's CPU step) on the full headline scene,
    `nsteps` steps from the same state."""
    om = load_oracle(tb)
    orc = om.Oracle(tb._abi)
    mesh, prm = sc.mesh, sc.params
    P = sc.particles.to("torch", device="cuda", dtype=np.float64)
    part = tb.Partition(mesh, P.n, backend="torch", device="cuda")
    G = tb.generate_grid(mesh, np.float64, backend="torch", device="cuda")
    runtime.step(G, P, part, mesh, prm, nsteps, ctx=ctx)
    ctx.synchronize()
    got = P.numpy()
    del P, part, G
    Pc = sc.particles.to("numpy")
    Gc = tb.generate_grid(mesh)
    t0 = time.perf_counter()
    orc.step_parallel(mesh, Pc, Gc, prm, nsteps, om.cores())
    cpu_s = time.perf_counter() - t0
    out = {"steps": nsteps, "n_particles": Pc.n, "oracle_threads": om.cores(), "oracle_s": cpu_s,
           "bound": 1e-9}
    for k in ("x", "v", "F", "sigma", "V"):
        ref = getattr(Pc, k)
        out[f"rel_err_{k}"] = float(np.linalg.norm(got[k] - ref) / np.linalg.norm(ref))
    out["pass"] = all(out[f"rel_err_{k}"] <= 1e-9 for k in ("x", "v", "F"))
    return out


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    tb = load_package()
    om = load_oracle(tb)
    oracle = om.Oracle(tb._abi)
    sc = tb.scenes.block_ordered(tb.scenes.cube3d(scale=args.scale))  # the order the B200 arm times
    mesh, prm = sc.mesh, sc.params
    P = sc.particles
    G = tb.generate_grid(mesh)
    threads = om.cores()
    for _ in range(args.warmup):
        oracle.step_parallel(mesh, P, G, prm, 1, threads)
    t0 = time.perf_counter()
    phases = oracle.step_parallel(mesh, P, G, prm, args.steps, threads)
    dt = time.perf_counter() - t0
    value = P.n * args.steps / dt
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded cube3d scene)",
        "config": {"workload": "cube3d: 256^3 cells, 16,777,216 particles, one MPM step per step",
                   "n_particles": P.n, "scale": args.scale, "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                         "sample": f"full workload, {args.steps} MPM steps after {args.warmup} warm-up, FP64, "
                                   "OpenMP colour-phased restatement of the reference CPU path",
                         "phase_s": dict(zip(["bin", "p2g", "grid", "g2p"], phases))},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--scale", type=int, default=1, help="shrink the cube scene (cells per axis / scale)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiable-rollout leg")
    ap.add_argument("--adj-scale", type=int, default=1, help="shrink the sphere scene of the adjoint leg")
    ap.add_argument("--no-taylor", action="store_true", help="skip the Taylor impact leg")
    ap.add_argument("--configs", default="clusters3d,sphere3d,dambreak3d",
                    help="comma list of the other configurations to measure (clusters3d, sphere3d, dambreak3d), "
                         "or 'none'")
    ap.add_argument("--config-scale", type=int, default=1, help="shrink the other configurations' scenes")
    ap.add_argument("--no-oracle-check", action="store_true", help="skip the full-size FP64 oracle check")
    ap.add_argument("--quick", action="store_true",
                    help="only the timed FP32 leg (for profiler captures); prints a reduced line")
    ap.add_argument("--kernel-case", default=None, metavar="SCENE:SCALE[:FORM][:adjoint]",
                    help="only this scene's steps (or its tape's backward pass), for per-kernel profiler captures")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    tb = load_package()
    from tesserae_b200 import runtime
    ctx = runtime.Context(local)

    if args.kernel_case:
        if rank == 0:
            print(json.dumps(kernel_case(tb, runtime, ctx, args.kernel_case, args.steps, args.warmup)), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    sc = tb.scenes.cube3d(scale=args.scale)
    mesh, prm = sc.mesh, sc.params
    host64 = sc.particles
    n = host64.n

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks_here(v: float) -> float:
        return max_over_ranks(v, dist, "cuda")

    def timed_steps(P, G, part, K):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        l0 = ctx.launches
        e0.record()
        runtime.step(G, P, part, mesh, prm, K, ctx=ctx)
        e1.record()
        barrier()
        return e0.elapsed_time(e1), ctx.launches - l0

    # The headline form with the particles in generation order (column-major
    # lattice), timed before they are put in block order for every other leg.
    gen_order = None
    if not args.quick:
        dtype, x64, _ = FORMS["x64"]
        P = host64.to("torch", device="cuda", dtype=dtype, x64=x64)
        part = tb.Partition(mesh, n, backend="torch", device="cuda")
        G = tb.generate_grid(mesh, dtype, backend="torch", device="cuda")
        runtime.step(G, P, part, mesh, prm, args.warmup, ctx=ctx)
        ctx.synchronize()
        score = runtime.block_ordered_particle_contiguity(part, n, ctx=ctx)
        ms, _ = timed_steps(P, G, part, args.steps)
        ms = max_over_ranks_here(ms)
        gen_order = {"value": job_throughput(world, n, args.steps, ms), "ms_per_step": ms / args.steps,
                     "contiguity": score,
                     "order": "generation order (column-major lattice), headline form"}
        del P, part, G
        torch.cuda.empty_cache()
    # reorder_particles! once after the first binning (docs/src/parallel.md:47-57)
    tb.scenes.block_ordered(sc)
    x0 = host64.x.copy()

    results = {}
    forms = ("x64",) if args.quick else ("x64", "f32", "f64")
    for name in forms:
        dtype, x64, _ = FORMS[name]
        P = host64.to("torch", device="cuda", dtype=dtype, x64=x64)
        part = tb.Partition(mesh, n, backend="torch", device="cuda")
        G = tb.generate_grid(mesh, dtype, backend="torch", device="cuda")
        runtime.step(G, P, part, mesh, prm, args.warmup, ctx=ctx)
        ctx.synchronize()
        with ClockSampler(local) as clk:
            ms, launches = timed_steps(P, G, part, args.steps)
        ms = max_over_ranks_here(ms)
        # per-kernel device time, profiled separately (events add launch gaps)
        ctx.profile(True)
        runtime.step(G, P, part, mesh, prm, 3, ctx=ctx)
        kt = ctx.profile_read()
        ctx.profile(False)
        results[name] = {"ms": ms, "launches": launches, "kernels": kt, "clocks": clk.summary()}
        del P, part, G
        torch.cuda.empty_cache()

    if args.quick:
        if rank == 0:
            hd = results["x64"]
            print(json.dumps({"metric": METRIC, "value": job_throughput(world, n, args.steps, hd["ms"]),
                              "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
                              "warmup": args.warmup, "ms_per_step": hd["ms"] / args.steps, "quick": True,
                              "kernels_ms_per_step": {k: v[1] / 3 for k, v in sorted(hd["kernels"].items())}}),
                  flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    # Both FP32 forms against the plain FP64 form after 100 steps of the same
    # scene (all on the device; the FP64 form is parity-tested against the
    # FP64 oracle).
    Ps = {}
    for name in ("x64", "f32", "f64"):
        dtype, x64, _ = FORMS[name]
        P = host64.to("torch", device="cuda", dtype=dtype, x64=x64)
        part = tb.Partition(mesh, n, backend="torch", device="cuda")
        G = tb.generate_grid(mesh, dtype, backend="torch", device="cuda")
        runtime.step(G, P, part, mesh, prm, sc.nsteps, ctx=ctx)
        ctx.synchronize()
        Ps[name] = {k: getattr(P, k).double().cpu().numpy() for k in ("x", "v")}
        del P, part, G
        torch.cuda.empty_cache()

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    def accuracy(name):
        a, b = Ps[name], Ps["f64"]
        return {"steps": sc.nsteps, "rel_err_x": rel(a["x"], b["x"]), "rel_err_v": rel(a["v"], b["v"]),
                "rel_err_displacement": rel(a["x"] - x0, b["x"] - x0),
                "against": "plain FP64 form on the device (parity-tested against the FP64 oracle)"}

    acc = accuracy("x64")
    acc_f32 = accuracy("f32")
    del Ps

    # End to end through the host-buffer C-ABI call: pinned host state in,
    # S MPM steps, state out, every call.
    S = 10
    calls = max(2, args.steps // S)
    hostp = host64.to("pinned", dtype=np.float32, x64=True)
    runtime.rollout_host(hostp, mesh, prm, S, ctx=ctx)  # allocates the context's device state
    barrier()
    t0 = time.perf_counter()
    for _ in range(calls):
        runtime.rollout_host(hostp, mesh, prm, S, ctx=ctx)
    barrier()
    e2e_s = max_over_ranks_here(time.perf_counter() - t0)
    # in: x, v, V, sigma, F (the step's inputs); out: the same and grad_v (written by every G2P)
    in_bytes = hostp.x.nbytes + hostp.v.nbytes + hostp.V.nbytes + hostp.sigma.nbytes + hostp.F.nbytes
    out_bytes = in_bytes + hostp.grad_v.nbytes
    e2e = {"value": job_throughput(world, n, S * calls, 1e3 * e2e_s), "unit": "particle-steps/s", "h2d_bytes_per_step": in_bytes,
           "d2h_bytes_per_step": out_bytes, "mpm_steps_per_call": S,
           "note": "one bench step = one tb_rollout_host_f32x64 call on pinned host buffers (H2D, S steps, D2H)"}
    del hostp

    # One MPM step per call: every step pays the whole state's round trip.
    hostp = host64.to("pinned", dtype=np.float32, x64=True)
    runtime.rollout_host(hostp, mesh, prm, 1, ctx=ctx)
    calls1 = 5
    barrier()
    t0 = time.perf_counter()
    for _ in range(calls1):
        runtime.rollout_host(hostp, mesh, prm, 1, ctx=ctx)
    barrier()
    e2e1_s = max_over_ranks_here(time.perf_counter() - t0)
    e2e["one_step_per_call"] = {"value": job_throughput(world, n, calls1, 1e3 * e2e1_s), "unit": "particle-steps/s",
                                "h2d_bytes_per_step": in_bytes, "d2h_bytes_per_step": out_bytes,
                                "mpm_steps_per_call": 1, "calls": calls1}
    del hostp

    peak, peak_src = measured_peaks()
    oracle_check = None
    if world == 1 and not args.no_oracle_check and args.scale == 1:
        oracle_check = fullsize_oracle_check(tb, runtime, ctx, sc)
    configs = {}
    # the other configurations and the oracle check run at N = 1 only
    wanted = [c for c in args.configs.split(",") if c and c != "none"] if world == 1 else []
    cs = args.config_scale
    for cname in wanted:
        if cname == "clusters3d":
            csc = tb.scenes.clusters3d(scale=cs)
            configs[cname] = config_leg(tb, runtime, ctx, csc, ("x64", "f64"), steps=10, warmup=3,
                                        acc_steps=csc.nsteps, peak=peak, per_particle=("m",), sparse_forms=("x64",))
            configs[cname]["workload"] = ("clusters3d: 512^3 cells, 64 Gaussian clusters (sigma 0.02), lognormal "
                                          "masses, Neo-Hookean E=1e5 nu=0.35, dt=2.5e-5; block order")
        elif cname == "sphere3d":
            csc = tb.scenes.block_ordered(tb.scenes.sphere3d(scale=cs))
            configs[cname] = config_leg(tb, runtime, ctx, csc, ("x64", "f64"), steps=20, warmup=3,
                                        acc_steps=csc.nsteps, peak=peak, per_particle=("mu", "lam"))
            configs[cname]["workload"] = ("sphere3d forward: 64^3 cells, sphere r=0.3, jittered 4^3 per cell, "
                                          "per-particle E, dt=5e-4; block order")
        elif cname == "dambreak3d":
            csc = tb.scenes.dambreak3d(scale=cs, particles=False)  # each form builds its own state on the device
            configs[cname] = config_leg(tb, runtime, ctx, csc, ("x64", "f32", "f64"), steps=5, warmup=3,
                                        acc_steps=csc.nsteps, peak=peak, apic=True)
            configs[cname]["workload"] = ("dambreak3d: 384^3 cells, column [0,0.4]x[0,1]x[0,0.8] at 2^3 per cell, "
                                          "WLS(uGIMP) + APIC, fluid K=2e6, slip walls, dt=2.5e-5; block order")
            if not args.no_adjoint:
                configs[cname]["adjoint_last_20"] = dambreak_adjoint_leg(tb, runtime, ctx)
        else:
            raise SystemExit(f"unknown config {cname}")

    adjoint = None if (args.no_adjoint or world > 1) else adjoint_leg(tb, runtime, ctx, scale=args.adj_scale)
    taylor = None if (args.no_taylor or rank != 0) else taylor_leg(tb, runtime, ctx)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    # Roofline of the dominant kernel of the headline form.
    kt = results["x64"]["kernels"]
    dom = max(("p2g", "g2p"), key=lambda k: kt.get(k, (0, 0.0))[1])
    launches_dom, ms_dom = kt[dom]
    per_p, per_n = algorithmic_bytes(dom, 4, 8)
    nact = active_nodes(mesh, host64.x)
    alg_bytes = n * per_p + nact * per_n
    achieved = alg_bytes / (ms_dom / launches_dom * 1e-3) / 1e9
    traffic = read_traffic(dom, n)
    sp, sn = step_bytes(4, 8)
    step_alg = n * sp + nact * sn
    hd = results["x64"]
    step_gbs = step_alg / (hd["ms"] / args.steps * 1e-3) / 1e9

    cpu = None
    if world == 1 and not args.no_cpu:
        om = load_oracle(tb)
        oracle = om.Oracle(tb._abi)
        cores = om.cores()
        Pc = host64.to("numpy")
        Gc = tb.generate_grid(mesh)
        oracle.step_parallel(mesh, Pc, Gc, prm, 1, cores)
        t0 = time.perf_counter()
        nst = 2
        oracle.step_parallel(mesh, Pc, Gc, prm, nst, cores)
        dt = time.perf_counter() - t0
        cpu = {"value": n * nst / dt, "unit": "particle-steps/s", "cores": cores, "kind": "port",
               "sample": f"cube3d full workload ({n} particles), {nst} MPM steps after 1 warm-up, FP64 "
                         "OpenMP colour-phased restatement of the reference CPU path"}

    f32, f64 = results["f32"], results["f64"]
    out = {
        "metric": METRIC,
        "value": job_throughput(world, n, args.steps, hd["ms"]),
        "unit": "particle-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": hd["ms"] / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded cube3d scene, numpy PCG64)",
        "config": {"workload": "cube3d: unit cube 256^3 cells, centre cube side 0.5 at 2^3 particles/cell, "
                               "Neo-Hookean E=1e6 nu=0.3, gravity, dt=5e-5; one MPM step per bench step",
                   "n_particles": n, "scale": args.scale, "form": FORMS["x64"][2],
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": "inputs larger than L2 (3.1 GB particle state per replica)",
                   "particle_order": "block order: reorder_particles! once after the first binning, as "
                                     "docs/src/parallel.md:47-57 sets up a GPU run (the reference arm and "
                                     "the CPU baseline time the same order; generation order under "
                                     "generation_order)"},
        "accuracy": dict(acc, fullsize_oracle_check=oracle_check),
        "configs": configs,
        "fp32_positions": {"value": job_throughput(world, n, args.steps, f32["ms"]), "ms_per_step": f32["ms"] / args.steps,
                           "form": FORMS["f32"][2], "accuracy": acc_f32},
        "fp64_plain": {"value": job_throughput(world, n, args.steps, f64["ms"]), "ms_per_step": f64["ms"] / args.steps},
        "generation_order": gen_order,
        "adjoint_over_forward": adjoint,
        "taylor_impact": taylor,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                     "algorithmic_bytes": alg_bytes, "bytes_per_particle": per_p, "bytes_per_active_node": per_n,
                     "active_nodes": nact},
        "step_roofline": {"bound": "hbm", "achieved": step_gbs, "peak": peak, "unit": "GB/s", "frac": step_gbs / peak,
                          "algorithmic_bytes": step_alg, "bytes_per_particle": sp, "bytes_per_active_node": sn},
        "kernels_ms_per_step": {k: v[1] / 3 for k, v in sorted(kt.items())},
        "kernels_ms_per_step_fp32_positions": {k: v[1] / 3 for k, v in sorted(f32["kernels"].items())},
        "kernels_ms_per_step_f64": {k: v[1] / 3 for k, v in sorted(f64["kernels"].items())},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": hd["launches"],
        "clocks": hd["clocks"],
    }
    print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
