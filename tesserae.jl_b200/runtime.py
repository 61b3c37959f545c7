"""Device API: the reference's hot-path verbs on torch device arrays, through the
C ABI of libtesserae_b200.so.

  update(weights, particles, mesh, params)      update!(weights, particles, mesh)      basis_weight.jl:714
  update(partition, particles, mesh, ctx)       update!(partition, particles.x)         gpu_block_strategy.jl:142
  P2G(grid, particles, partition, mesh, params) @P2G (m, mv, f sums + grid half)        p2g.jl:66, gpu.jl:196
  G2P(grid, particles, mesh, params)            @G2P (FLIP/APIC + Neo-Hookean)          g2p.jl:71, gpu.jl:226
  step(...)                                     the whole README.md:66-87 loop body, n times
  reorder_particles(particles, partition, thr)  reorder_particles!                      gpu_block_strategy.jl:194
  adjoint_step / tape_forward / tape_backward   reverse mode (no reference counterpart)
  rollout_grad                                  gradients of a rollout loss w.r.t. v0 and log E

The precision form follows the particle dtype: float64 -> the plain `_f64`
entry points, float32 (F float64) -> the mixed `_f32` ones, float32 with
float64 positions (`Particles(..., x64=True)`) -> `tb_step_f32x64` /
`tb_rollout_host_f32x64` (step and rollout_host only). Every call raises
RuntimeError with the library's message on a non-zero status; there is no
fallback path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .state import Adjoint, BasisWeights, CartesianMesh, Grid, Particles, Partition


def _suffix(dtype) -> str:
    dt = np.dtype(dtype)
    if dt == np.float64:
        return "f64"
    if dt == np.float32:
        return "f32"
    raise TypeError(f"unsupported scalar type {dt}")


class Context:
    """A tb_ctx bound to one device and stream (default: torch's current stream)."""

    def __init__(self, device: int = 0, stream=None):
        import torch
        self.lib = _abi.load_library()
        if stream is None:
            stream = torch.cuda.current_stream(device)
        self.stream = stream
        handle = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream or 0)
        self.ptr = self.lib.tb_create(int(device), C.c_void_p(handle))
        if not self.ptr:
            raise RuntimeError("tb_create failed (no CUDA device?)")
        self.device = device

    def close(self):
        if getattr(self, "ptr", None):
            self.lib.tb_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int, what: str):
        if rc != _abi.TB_OK:
            msg = self.lib.tb_last_error(self.ptr)
            raise RuntimeError(f"{what}: status {rc}: {msg.decode() if msg else ''}")

    def synchronize(self):
        self.check(self.lib.tb_synchronize(self.ptr), "tb_synchronize")

    @property
    def launches(self) -> int:
        return int(self.lib.tb_launch_count(self.ptr))

    def profile(self, on: bool = True):
        """Enable/disable per-kernel CUDA-event timing of this library's launches."""
        self.check(self.lib.tb_profile_enable(self.ptr, int(bool(on))), "tb_profile_enable")

    def profile_read(self) -> dict:
        """{kernel family: (launches, ms)} accumulated since the last read (synchronises)."""
        cap = 64
        buf = (_abi.tb_kernel_time * cap)()
        cnt = C.c_int32()
        self.check(self.lib.tb_profile_read(self.ptr, buf, cap, C.byref(cnt)), "tb_profile_read")
        return {buf[i].name.decode(): (int(buf[i].launches), float(buf[i].ms)) for i in range(min(cnt.value, cap))}

    def release_tape(self):
        """Free this context's tape buffers (the next tape_forward allocates again)."""
        self.check(self.lib.tb_tape_release(self.ptr), "tb_tape_release")

    def fn(self, name: str, dtype):
        return getattr(self.lib, f"{name}_{_suffix(dtype)}")

    def pfn(self, name: str, particles: Particles, x64_ok: bool = False):
        """Entry point for the particles' precision form."""
        if getattr(particles, "x64", False):
            if not x64_ok:
                raise TypeError(f"{name}: the FP64-position form is available for step and rollout_host only")
            return getattr(self.lib, f"{name}_f32x64")
        return self.fn(name, particles.dtype)


def _ref(s):
    return C.byref(s)


def update(target, particles: Particles, mesh: CartesianMesh, params=None, ctx: Context | None = None):
    """update!(weights, particles, mesh) or update!(partition, particles.x)."""
    ctx = ctx or _default()
    if isinstance(target, BasisWeights):
        if params is None:
            raise ValueError("update(weights, ...) needs step params (basis kind, uGIMP length)")
        rc = ctx.pfn("tb_update_weights", particles)(ctx.ptr, _ref(mesh.struct()), _ref(particles.struct()),
                                                          _ref(params), _ref(target.struct()))
        ctx.check(rc, "update!(weights)")
        return target
    if isinstance(target, Partition):
        na, nass = C.c_int64(), C.c_int64()
        # binning reads only x: FP64 positions bin by the Float64 rule
        xdtype = np.float64 if getattr(particles, "x64", False) else particles.dtype
        rc = ctx.fn("tb_bin_particles", xdtype)(ctx.ptr, _ref(mesh.struct()), _ref(particles.struct()),
                                                _ref(target.struct()), C.byref(na), C.byref(nass))
        ctx.check(rc, "update!(partition)")
        target.nactive, target.nassigned = na.value, nass.value
        return target
    raise TypeError(f"update: unsupported target {type(target).__name__}")


def P2G(grid: Grid, particles: Particles, partition: Partition, mesh: CartesianMesh, params,
        grid_half: bool = True, ctx: Context | None = None):
    """The recognised @P2G body: m = sum w m_p, mv = sum w m_p v_p (APIC: + B D^-1 (x_i - x_p)),
    f = sum -V sigma grad w + w m_p g; with `grid_half`, vn = mv/m and v = vn + dt f/m."""
    ctx = ctx or _default()
    rc = ctx.pfn("tb_p2g", particles)(ctx.ptr, _ref(mesh.struct()), _ref(particles.struct()),
                                           _ref(partition.struct()), _ref(grid.struct()), _ref(params))
    ctx.check(rc, "@P2G")
    if grid_half:
        rc = ctx.fn("tb_grid_update", particles.dtype)(ctx.ptr, _ref(mesh.struct()), _ref(grid.struct()),
                                                       _ref(params))
        ctx.check(rc, "@P2G grid half")
    return grid


def G2P(grid: Grid, particles: Particles, mesh: CartesianMesh, params, ctx: Context | None = None):
    """The recognised @G2P body (README.md:79-86 / APIC)."""
    ctx = ctx or _default()
    rc = ctx.pfn("tb_g2p", particles)(ctx.ptr, _ref(mesh.struct()), _ref(grid.struct()),
                                           _ref(particles.struct()), _ref(params))
    ctx.check(rc, "@G2P")
    return particles


def update_sparsity(grid: Grid, particles: Particles, partition: Partition, mesh: CartesianMesh,
                    ctx: Context | None = None, headroom: float = 1.0) -> int:
    """update_sparsity!(grid, particles.x) for a sparse grid (src/Grids/sparsity.jl:19-60):
    bins the particles into `partition`, numbers the node blocks within one block
    of a block that holds particles, zero-fills the stored fields, and returns
    the number of stored nodes per field. The field arrays grow (to the count
    times `headroom`) when they are too small."""
    ctx = ctx or _default()
    if not grid.sparse:
        raise TypeError("update_sparsity needs a sparse grid (generate_grid(..., sparse=True))")
    n = C.c_int64(0)
    fn = ctx.pfn("tb_update_sparsity", particles, x64_ok=True)
    rc = fn(ctx.ptr, _ref(mesh.struct()), _ref(particles.struct()), _ref(partition.struct()), _ref(grid.struct()),
            C.byref(n))
    need = int(n.value)
    if rc == _abi.TB_ERR_CAPACITY or need * headroom > grid.capacity:
        grid.reserve(int(need * max(headroom, 1.0)))
        rc = fn(ctx.ptr, _ref(mesh.struct()), _ref(particles.struct()), _ref(partition.struct()),
                _ref(grid.struct()), C.byref(n))
    ctx.check(rc, "update_sparsity")
    return need


def step(grid: Grid, particles: Particles, partition: Partition, mesh: CartesianMesh, params, nsteps: int = 1,
         ctx: Context | None = None, reorder_threshold: float | None = None, sparse_headroom: float = 1.5):
    """`nsteps` fused steps (bin -> P2G -> grid update -> G2P) without host sync.
    With `reorder_threshold`, every binning is followed by
    `reorder_particles!(particles, partition; threshold=reorder_threshold)`,
    decided on the device. A sparse grid follows the particles (its sparsity is
    updated at every step on the device); its field arrays are first sized for
    the current positions times `sparse_headroom`, and a step whose active
    blocks would exceed them is reported as a device error."""
    ctx = ctx or _default()
    if grid.sparse:
        update_sparsity(grid, particles, partition, mesh, ctx=ctx, headroom=sparse_headroom)
    if reorder_threshold is None:
        rc = ctx.pfn("tb_step", particles, x64_ok=True)(ctx.ptr, _ref(mesh.struct()), _ref(particles.struct()),
                                                        _ref(partition.struct()), _ref(grid.struct()), _ref(params),
                                                        int(nsteps))
    else:
        rc = ctx.pfn("tb_step_reorder", particles, x64_ok=True)(
            ctx.ptr, _ref(mesh.struct()), _ref(particles.struct()), _ref(partition.struct()), _ref(grid.struct()),
            _ref(params), int(nsteps), float(reorder_threshold))
    ctx.check(rc, "step")


def g2p2g(grid: Grid, particles: Particles, partition: Partition, mesh: CartesianMesh, params,
          ctx: Context | None = None):
    """@G2P2G (src/Transfer/g2p2g.jl) for the FLIP/PIC equation set: each
    particle's G2P, then its P2G of m, mv, f with the weights of its position
    before the G2P moved it, then the grid half; binned into `partition` first."""
    ctx = ctx or _default()
    rc = ctx.pfn("tb_g2p2g", particles, x64_ok=True)(ctx.ptr, _ref(mesh.struct()), _ref(particles.struct()),
                                                     _ref(partition.struct()), _ref(grid.struct()), _ref(params))
    ctx.check(rc, "g2p2g")


def max_wave_speed(particles: Particles, params, ctx: Context | None = None) -> float:
    """max over the particles of sqrt((lambda + 2 mu) / (m / V)) + |v|, reduced
    on the device (the speed of the Taylor impact's time step)."""
    ctx = ctx or _default()
    out = C.c_double()
    fn = ctx.fn("tb_max_wave_speed", particles.dtype)
    ctx.check(fn(ctx.ptr, int(particles.dim), _ref(particles.struct()), _ref(params), C.byref(out)),
              "max_wave_speed")
    return float(out.value)


def adaptive_steps(grid: Grid, particles: Particles, partition: Partition, mesh: CartesianMesh, params,
                   nsteps: int, cfl: float = 0.8, ctx: Context | None = None) -> float:
    """`nsteps` steps of the Taylor impact's loop (docs/src/gpu.md:281-360):
    each step takes dt = cfl h / max c from the particles' current state
    (max_wave_speed, one device reduction and host read per step, as the
    reference's `maximum(particles.c)`), then runs one step. Returns the time
    advanced."""
    ctx = ctx or _default()
    prm = type(params).from_buffer_copy(params)
    t = 0.0
    for _ in range(int(nsteps)):
        prm.dt = cfl * mesh.h / max_wave_speed(particles, prm, ctx=ctx)
        step(grid, particles, partition, mesh, prm, 1, ctx=ctx)
        t += prm.dt
    return t


def reorder_particles(particles: Particles, partition: Partition, threshold: float = 1.0,
                      ctx: Context | None = None) -> bool:
    """reorder_particles!(particles, partition; threshold) (src/Parallel/gpu_block_strategy.jl:194-202):
    permute every particle field into the partition's block order when the
    contiguity score is below `threshold`; returns whether it reordered."""
    ctx = ctx or _default()
    done = C.c_int32()
    rc = ctx.pfn("tb_reorder_particles", particles, x64_ok=True)(ctx.ptr, int(particles.dim), _ref(particles.struct()),
                                                                 _ref(partition.struct()), float(threshold),
                                                                 C.byref(done))
    ctx.check(rc, "reorder_particles!")
    return bool(done.value)


def block_ordered_particle_contiguity(partition: Partition, n: int, ctx: Context | None = None) -> float:
    """Tesserae.block_ordered_particle_contiguity (src/Parallel/gpu_block_strategy.jl:172-191)."""
    ctx = ctx or _default()
    score = C.c_double()
    ctx.check(ctx.lib.tb_particle_contiguity(ctx.ptr, _ref(partition.struct()), int(n), C.byref(score)),
              "block_ordered_particle_contiguity")
    return float(score.value)


def rollout_host(particles: Particles, mesh: CartesianMesh, params, nsteps: int, ctx: Context | None = None):
    """Host-buffer rollout: `particles` holds numpy arrays; state is copied in,
    advanced `nsteps` steps on the device and copied back (synchronous)."""
    ctx = ctx or _default()
    if particles.backend not in ("numpy", "pinned"):
        raise TypeError("rollout_host takes host (numpy or pinned) particles")
    rc = ctx.pfn("tb_rollout_host", particles, x64_ok=True)(ctx.ptr, _ref(mesh.struct()),
                                                            _ref(particles.struct()), _ref(params), int(nsteps))
    ctx.check(rc, "rollout_host")


def adjoint_step(grid: Grid, particles: Particles, partition: Partition, mesh: CartesianMesh, params,
                 adj: Adjoint, ctx: Context | None = None):
    """One step backwards: `particles` is the state at the start of the step;
    `adj` (float64 device arrays) maps end-of-step sensitivities to start-of-step
    ones in place (mu / lam accumulate)."""
    ctx = ctx or _default()
    rc = ctx.pfn("tb_adjoint_step", particles, x64_ok=True)(ctx.ptr, _ref(mesh.struct()), _ref(particles.struct()),
                                                    _ref(partition.struct()), _ref(grid.struct()), _ref(params),
                                                    _ref(adj.struct()))
    ctx.check(rc, "adjoint_step")


def tape_bytes(mesh: CartesianMesh, n: int, dtype, nsteps: int, checkpoint_every: int, apic: bool = False,
               x64: bool = False) -> int:
    """Device bytes a tape holds (forward and backward pass) for `n` particles of
    element type `dtype` (with FP64 positions if `x64`) over `nsteps` steps,
    checkpointed every `checkpoint_every` steps (1: the whole tape, no recompute
    in the backward)."""
    lib = _abi.load_library()
    b = int(lib.tb_tape_bytes(C.byref(mesh.struct()), int(n), int(np.dtype(dtype).itemsize), int(bool(apic)),
                              int(bool(x64)), int(nsteps), int(checkpoint_every)))
    if b < 0:
        raise ValueError("tape_bytes: invalid arguments")
    return b


def tape_slot_bytes(mesh: CartesianMesh, n: int, dtype, apic: bool = False, x64: bool = False) -> int:
    """Device bytes one step of the whole tape holds (state, grid, partition)."""
    return tape_bytes(mesh, n, dtype, 1, 1, apic, x64)


def choose_checkpoint_every(mesh: CartesianMesh, n: int, dtype, nsteps: int, apic: bool = False,
                            device=None, budget: float = 0.6, fallback: int = 20, x64: bool = False) -> int:
    """1 (the whole tape in device memory) when it takes at most `budget` of the
    device's free memory, else `fallback`."""
    import torch
    free, _ = torch.cuda.mem_get_info(device)
    return 1 if tape_bytes(mesh, n, dtype, nsteps, 1, apic, x64) <= budget * free else fallback


def tape_forward(grid: Grid, particles: Particles, partition: Partition, mesh: CartesianMesh, params,
                 nsteps: int, checkpoint_every: int = 20, ctx: Context | None = None):
    """Advance `nsteps` steps (as `step`) keeping checkpoints every
    `checkpoint_every` steps; 1 keeps every step's state, grid and partition (the
    whole tape), so tape_backward runs no forward step."""
    ctx = ctx or _default()
    rc = ctx.pfn("tb_tape_forward", particles, x64_ok=True)(ctx.ptr, _ref(mesh.struct()), _ref(particles.struct()),
                                                    _ref(partition.struct()), _ref(grid.struct()), _ref(params),
                                                    int(nsteps), int(checkpoint_every))
    ctx.check(rc, "tape_forward")


def tape_backward(grid: Grid, particles: Particles, partition: Partition, mesh: CartesianMesh, params,
                  adj: Adjoint, ctx: Context | None = None):
    """Sensitivities to the final state (in `adj`) -> sensitivities to the step-0
    state; `particles` is restored to the step-0 state."""
    ctx = ctx or _default()
    rc = ctx.pfn("tb_tape_backward", particles, x64_ok=True)(ctx.ptr, _ref(mesh.struct()), _ref(particles.struct()),
                                                     _ref(partition.struct()), _ref(grid.struct()), _ref(params),
                                                     _ref(adj.struct()))
    ctx.check(rc, "tape_backward")


def rollout_grad(particles: Particles, mesh: CartesianMesh, params, nsteps: int, loss_grad,
                 checkpoint_every: int | None = None, nu: float | None = None, ctx: Context | None = None):
    """Gradients of a rollout loss with respect to the initial velocities and the
    per-particle log Young's modulus.

    `loss_grad(particles_final) -> (loss, dL/dx, dL/dv)` gives the loss and its
    sensitivities to the final positions and velocities (float64 tensors of
    shape (dim, n)). With per-particle Lame arrays (particles.mu / particles.lam)
    and E entering both as mu = E / (2 (1 + nu)), lambda = E nu / ((1 + nu)(1 - 2 nu)),
    dL/dlogE = mu dL/dmu + lambda dL/dlambda. `particles` is left in its initial
    state. `checkpoint_every` None: the whole tape when it fits in device memory
    (choose_checkpoint_every). Returns (loss, dL/dv0, dL/dlogE or None)."""
    import torch
    ctx = ctx or _default()
    D, n = particles.dim, particles.n
    if checkpoint_every is None:
        checkpoint_every = choose_checkpoint_every(mesh, n, particles.dtype, nsteps,
                                                   params.transfer == _abi.TB_TRANSFER_APIC, particles.device,
                                                   x64=getattr(particles, "x64", False))
    part = Partition(mesh, n, backend="torch", device=particles.device or "cuda")
    grid = Grid(mesh, particles.dtype, backend="torch", device=particles.device or "cuda")
    tape_forward(grid, particles, part, mesh, params, nsteps, checkpoint_every, ctx=ctx)
    loss, gx, gv = loss_grad(particles)
    lame = particles.mu is not None and particles.lam is not None
    apic = params.transfer == _abi.TB_TRANSFER_APIC
    adj = Adjoint(n, D, backend="torch", device=particles.device or "cuda", lame=lame, apic=apic)
    adj.x.copy_(gx)
    adj.v.copy_(gv)
    tape_backward(grid, particles, part, mesh, params, adj, ctx=ctx)
    glogE = None
    if lame:
        glogE = adj.mu * particles.mu.double() + adj.lam * particles.lam.double()
    torch.cuda.current_stream().synchronize()
    return loss, adj.v, glogE


class RolloutFunction:
    """torch.autograd.Function over the checkpointed rollout: forward maps the
    initial velocities (dim, n) to the final positions (dim, n); backward runs the
    adjoint tape. The counterpart of a ChainRulesCore rrule on the Julia side."""

    @staticmethod
    def apply(v0, particles: Particles, mesh: CartesianMesh, params, nsteps: int, checkpoint_every: int | None = None,
              ctx: Context | None = None):
        import torch
        if checkpoint_every is None:
            checkpoint_every = choose_checkpoint_every(mesh, particles.n, particles.dtype, nsteps,
                                                       params.transfer == _abi.TB_TRANSFER_APIC, v0.device,
                                                       x64=getattr(particles, "x64", False))

        class _F(torch.autograd.Function):
            @staticmethod
            def forward(fctx, v):
                c = ctx or _default()
                particles.v.copy_(v.to(particles.v.dtype))
                fctx.part = Partition(mesh, particles.n, backend="torch", device=v.device)
                fctx.grid = Grid(mesh, particles.dtype, backend="torch", device=v.device)
                tape_forward(fctx.grid, particles, fctx.part, mesh, params, nsteps, checkpoint_every, ctx=c)
                xT = particles.x.detach().double().clone()
                return xT

            @staticmethod
            def backward(fctx, gx):
                c = ctx or _default()
                adj = Adjoint(particles.n, particles.dim, backend="torch", device=gx.device, lame=False,
                              apic=params.transfer == _abi.TB_TRANSFER_APIC)
                adj.x.copy_(gx.double())
                tape_backward(fctx.grid, particles, fctx.part, mesh, params, adj, ctx=c)
                return adj.v.to(v0.dtype)

        return _F.apply(v0)


_ctx = None


def _default() -> Context:
    global _ctx
    if _ctx is None:
        _ctx = Context()
    return _ctx
