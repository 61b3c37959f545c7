"""Z-slab decomposition of the explicit MPM step over ranks (one rank per GPU).

Each rank owns a block-aligned range of cells [c0, c1) along the last axis and
the particles whose cell lies in it. It runs the step on a local mesh that
covers its cells plus `HALO` = 2 node layers on each side (clipped at the
domain), so every owned particle's support window fits unclipped: a quadratic
B-spline or uGIMP (l <= h) window of a particle in cell c spans nodes c - 1 ..
c + 2, so the particles of rank r touch nodes [c0 - 1, c1 + 1] and those of two
neighbouring ranks share the three node layers [c - 1, c + 1] around their
common face c. Per step:

  1. P2G of the owned particles into the local grid (m, mv, f; zeroed first);
  2. one sum-exchange with each neighbour: the 3 shared layers of m, mv, f go
     both ways and are added, so both ranks hold the complete sums there (the
     only data-path collective; torch.distributed send/recv, NCCL over
     NVLink / NVSwitch on GPUs, gloo on CPU);
  3. the grid half on the whole local grid (the shared layers are identical on
     both ranks, so no second exchange is needed); slip walls of the last axis
     are applied by the ranks at the domain ends only;
  4. G2P of the owned particles;
  5. migration: particles whose new cell left [c0, c1) go to the neighbour
     (the CFL condition keeps a particle within one slab of cells per step,
     and slabs are at least one block, 4 cells, thick), every field moved
     alike; particles outside the domain stay where they are (block 0).

The compute of each phase comes from a `backend` with the methods
`p2g(mesh, particles, grid, params)`, `grid_update(mesh, grid, params)` and
`g2p(mesh, grid, particles, params)` on host (numpy) or device (torch) state;
`DeviceBackend` calls libtesserae_b200. The local mesh repeats the global node
coordinates exactly when `xmin + n0 h` is exact (power-of-two spacings with a
zero origin, as in the seeded scenes); otherwise they agree to rounding.

No kernel waits on another rank and no TMA or bulk copy is involved: the
exchange is a host-driven send/recv of contiguous node layers.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from .state import CartesianMesh, Grid, Particles

HALO = 2  # node layers beyond the owned cells on each side
SHARED = 3  # node layers two neighbouring ranks both touch (c - 1 .. c + 1 around a face c)


@dataclass
class SlabLayout:
    """Cells [c0, c1) of the last axis owned by `rank` of `world`, the local
    mesh and where its nodes sit in the global node numbering."""

    mesh: CartesianMesh
    world: int
    rank: int
    c0: int = 0
    c1: int = 0
    n0: int = 0  # first global node layer of the local mesh
    n1: int = 0  # one past the last
    local: CartesianMesh = None

    def __post_init__(self):
        m = self.mesh
        ax = m.dim - 1
        ncell = m.n_nodes[ax] - 1
        bw = 1 << m.block_size_log2
        nblk = -(-ncell // bw)
        if nblk < self.world:
            raise ValueError(f"slabs: {nblk} blocks along the last axis for {self.world} ranks")
        b0 = self.rank * nblk // self.world
        b1 = (self.rank + 1) * nblk // self.world
        self.c0, self.c1 = b0 * bw, min(b1 * bw, ncell)
        self.n0 = max(self.c0 - HALO, 0)
        self.n1 = min(self.c1 + HALO, ncell) + 1
        lims = [tuple(l) for l in m.lims]
        z0 = m.xmin[ax] + self.n0 * m.h
        z1 = m.xmin[ax] + (self.n1 - 1) * m.h
        lims[ax] = (z0, z1)
        self.local = CartesianMesh(m.h, *lims, block_size_log2=m.block_size_log2)
        assert self.local.n_nodes[ax] == self.n1 - self.n0

    def cell(self, x_last) -> np.ndarray:
        """Global cell index along the last axis of positions `x_last`, clamped
        into the domain: a particle outside the mesh belongs to the slab it is
        nearest (it is binned to block 0 there and moved by G2P's outside pass)."""
        m = self.mesh
        ax = m.dim - 1
        c = np.floor((np.asarray(x_last, dtype=np.float64) - m.xmin[ax]) * m.h_inv)
        return np.clip(c, 0, m.n_nodes[ax] - 2).astype(np.int64)

    def owns(self, x_last) -> np.ndarray:
        c = self.cell(x_last)
        return (c >= self.c0) & (c < self.c1)

    def shared_layers(self, side: int) -> tuple[int, int] | None:
        """Local node layers [a, b) shared with the neighbour below (side -1) or
        above (+1), or None at the domain end."""
        if side < 0:
            if self.rank == 0:
                return None
            a = self.c0 - 1 - self.n0
        else:
            if self.rank == self.world - 1:
                return None
            a = self.c1 - 1 - self.n0
        return a, a + SHARED

    def params(self, params):
        """`params` with the slip walls of the last axis kept only at the domain ends."""
        p = type(params).from_buffer_copy(params)
        ax = self.mesh.dim - 1
        if self.rank > 0:
            p.wall_mask &= ~(1 << (2 * ax))
        if self.rank < self.world - 1:
            p.wall_mask &= ~(1 << (2 * ax + 1))
        return p


def _layers(a, mesh: CartesianMesh, rng: tuple[int, int]):
    """View of node layers [rng) of the last axis of a grid field (..., nnodes)."""
    shape = a.shape[:-1] + tuple(reversed(mesh.n_nodes))  # column-major nodes: last axis slowest
    return a.reshape(shape)[..., rng[0]:rng[1], :, :] if mesh.dim == 3 else a.reshape(shape)[..., rng[0]:rng[1], :]


def _is_torch(a) -> bool:
    return not isinstance(a, np.ndarray)


def exchange_shared(layout: SlabLayout, grid: Grid, dist) -> None:
    """Step 2: add the neighbours' partial sums of m, mv, f on the shared node
    layers (both directions at once; every rank posts its sends and receives
    in the same order)."""
    import torch
    fields = [grid.m[None], grid.mv, grid.f]
    reqs, recvs = [], []
    for side in (-1, 1):
        rng = layout.shared_layers(side)
        if rng is None:
            continue
        peer = layout.rank + side
        parts = [_layers(f, layout.local, rng) for f in fields]
        if _is_torch(grid.m):
            send = torch.cat([p.reshape(-1) for p in parts]).contiguous()
        else:
            send = torch.from_numpy(np.concatenate([p.reshape(-1) for p in parts]).copy())
        recv = torch.empty_like(send)
        reqs.append(dist.isend(send, peer))
        reqs.append(dist.irecv(recv, peer))
        recvs.append((parts, recv))
    for r in reqs:
        r.wait()
    for parts, recv in recvs:
        off = 0
        for p in parts:
            k = p.numel() if _is_torch(p) else p.size
            add = recv[off:off + k].reshape(p.shape)
            if _is_torch(p):
                p += add
            else:
                p += add.numpy()
            off += k


def migrate(layout: SlabLayout, P: Particles, ids, dist):
    """Step 5: send the particles that left [c0, c1) to the neighbour whose
    slab holds them, receive the ones that entered; returns the new
    (particles, ids). `ids` (int64) travel with the particles."""
    import torch
    torch_state = _is_torch(P.x)
    dev = P.x.device if torch_state else "cpu"  # counts travel where the state lives (NCCL: the GPU)
    if torch_state and isinstance(ids, np.ndarray):
        ids = torch.from_numpy(ids).to(dev)
    x_last = P.x[-1].double().cpu().numpy() if torch_state else P.x[-1]
    cell = layout.cell(x_last)
    down = cell < layout.c0
    up = cell >= layout.c1
    below = SlabLayout(layout.mesh, layout.world, layout.rank - 1) if layout.rank > 0 else None
    above = SlabLayout(layout.mesh, layout.world, layout.rank + 1) if layout.rank < layout.world - 1 else None
    if (below is not None and (cell < below.c0).any()) or (above is not None and (cell >= above.c1).any()):
        raise RuntimeError("slabs.migrate: a particle moved past the neighbouring slab in one step")
    keep = ~(down | up)
    fields = [k for k in P.FIELDS if getattr(P, k) is not None]

    def sel(a, mask):
        if torch_state:
            return a[..., torch.from_numpy(mask).to(a.device)]
        return a[..., mask]

    outgoing = {-1: down, 1: up}
    incoming = {}
    for side in (-1, 1):
        peer = layout.rank + side
        if peer < 0 or peer >= layout.world:
            continue
        cnt = torch.tensor([int(outgoing[side].sum())], dtype=torch.int64, device=dev)
        rcnt = torch.empty(1, dtype=torch.int64, device=dev)
        rq = [dist.isend(cnt, peer), dist.irecv(rcnt, peer)]
        for r in rq:
            r.wait()
        incoming[side] = int(rcnt.item())
    # per field: one send and one receive per neighbour (the same order on every rank)
    new = {}
    for k in fields + ["ids"]:
        a = ids if k == "ids" else getattr(P, k)
        parts = [sel(a, keep)]
        for side in (-1, 1):
            if side not in incoming:
                continue
            peer = layout.rank + side
            out = sel(a, outgoing[side])
            send = out if torch_state else torch.from_numpy(np.ascontiguousarray(out))
            send = send.contiguous()
            shape = tuple(send.shape[:-1]) + (incoming[side],)
            recv = torch.empty(shape, dtype=send.dtype, device=send.device)
            rq = [dist.isend(send, peer), dist.irecv(recv, peer)]
            for r in rq:
                r.wait()
            parts.append(recv if torch_state else recv.numpy())
        new[k] = torch.cat(parts, dim=-1) if torch_state else np.concatenate(parts, axis=-1)
    n = new["x"].shape[-1]
    opt = tuple(k for k in P.OPTIONAL if getattr(P, k) is not None)
    Q = Particles(n, P.dim, P.dtype, backend=P.backend, device=P.device, optional=opt, x64=P.x64)
    for k in fields:
        dst = getattr(Q, k)
        if torch_state:
            dst.copy_(new[k])
        else:
            dst[...] = new[k]
    return Q, new["ids"]


def step(layout: SlabLayout, backend, P: Particles, ids, grid: Grid, params, dist, nsteps: int = 1):
    """`nsteps` steps of the decomposed MPM step on this rank (the same calls in
    the same order on every rank). Returns the new (particles, ids); `grid` is
    the rank's local grid (`generate_grid(layout.local, ...)`)."""
    prm = layout.params(params)
    for _ in range(nsteps):
        backend.p2g(layout.local, P, grid, prm)
        exchange_shared(layout, grid, dist)
        backend.grid_update(layout.local, grid, prm)
        backend.g2p(layout.local, grid, P, prm)
        P, ids = migrate(layout, P, ids, dist)
    return P, ids


def scatter(layout: SlabLayout, P: Particles):
    """This rank's share of a global particle state (host or device) and the
    global ids of those particles."""
    x_last = P.x[-1] if isinstance(P.x, np.ndarray) else P.x[-1].double().cpu().numpy()
    mine = layout.owns(x_last)
    idx = np.nonzero(mine)[0]
    opt = tuple(k for k in P.OPTIONAL if getattr(P, k) is not None)
    Q = Particles(len(idx), P.dim, P.dtype, backend=P.backend, device=P.device, optional=opt, x64=P.x64)
    for k in P.FIELDS:
        a = getattr(P, k)
        if a is None:
            continue
        if isinstance(a, np.ndarray):
            getattr(Q, k)[...] = a[..., idx]
        else:
            import torch
            getattr(Q, k).copy_(a[..., torch.from_numpy(idx).to(a.device)])
    return Q, idx.astype(np.int64)


class DeviceBackend:
    """The phases on device state through libtesserae_b200 (binning into the
    rank's own partition before each P2G)."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.part = None

    def p2g(self, mesh, P, grid, params):
        import copy
        from . import runtime
        from .state import Partition
        if self.part is None or len(self.part.blockids) < P.n:
            self.part = Partition(mesh, max(int(P.n * 1.25), 1), backend="torch", device=P.device or "cuda")
        view = copy.copy(self.part)  # this step's particle count; block arrays shared
        view.blockids = self.part.blockids[:P.n]
        view.particleindices = self.part.particleindices[:P.n]
        runtime.update(view, P, mesh, ctx=self.ctx)
        runtime.P2G(grid, P, view, mesh, params, grid_half=False, ctx=self.ctx)

    def grid_update(self, mesh, grid, params):
        fn = self.ctx.fn("tb_grid_update", grid.dtype)
        self.ctx.check(fn(self.ctx.ptr, C.byref(mesh.struct()), C.byref(grid.struct()), C.byref(params)),
                       "grid update")

    def g2p(self, mesh, grid, P, params):
        from . import runtime
        runtime.G2P(grid, P, mesh, params, ctx=self.ctx)
