"""Host-side mirror of the reference's data model for the explicit MPM path.

`CartesianMesh`, `generate_grid`, `generate_particles`, `generate_basis_weights`
and `Partition` follow the reference's surface (src/Mesh/cartesian.jl:38-102,
src/Grids/grid.jl:70-78, src/particles.jl:112-118, src/Basis/basis_weight.jl:413-432,
src/Parallel/partition.jl:37-56). Arrays are structure-of-arrays: every vector or
tensor field is one (ncomp, n) array whose rows are the component arrays the
C ABI takes, so `particles.x[d]` is the d-th coordinate of every particle.

Arrays are numpy arrays (host) or torch tensors (device); the same container
feeds the CUDA library (device) and the CPU oracle (host).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi


def _ptr(a) -> int | None:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    assert a.is_contiguous()
    return a.data_ptr()


def _row_ptrs(a, k: int) -> list[int | None]:
    """Pointers to rows 0..k-1 of a (k, n) array."""
    if a is None:
        return [None] * k
    if isinstance(a, np.ndarray):
        return [a[i].ctypes.data for i in range(k)]
    return [a[i].data_ptr() for i in range(k)]


# ---------------------------------------------------------------------------
# mesh
# ---------------------------------------------------------------------------

@dataclass
class CartesianMesh:
    """Uniform Cartesian mesh (src/Mesh/cartesian.jl:38-102).

    `CartesianMesh(h, (xmin, xmax), (ymin, ymax), ...)`: nodes per axis follow
    `_covered_axis` (:77-87): an axis whose length is not a multiple of h is
    extended by one node. `h_inv` is stored as the FP64 inverse, as the reference
    does (`T(inv(h))`).
    """

    h: float
    lims: tuple
    block_size_log2: int = 2
    n_nodes: tuple = field(init=False)
    xmin: tuple = field(init=False)
    h_inv: float = field(init=False)

    def __init__(self, h, *lims, block_size_log2=None):
        self.h = float(h)
        self.lims = tuple((float(a), float(b)) for a, b in lims)
        dim = len(self.lims)
        if dim not in (2, 3):
            raise ValueError("CartesianMesh: only 2D and 3D meshes are on the B200 path")
        if block_size_log2 is None:
            block_size_log2 = 2 if dim == 3 else 3
        self.block_size_log2 = int(block_size_log2)
        n = []
        for a, b in self.lims:
            if not a < b:
                raise ValueError("CartesianMesh: xmin must be < xmax")
            q = (b - a) / self.h
            k = round(q)
            if math.isclose(k, q, rel_tol=1e-12, abs_tol=1e-12):
                n.append(int(k) + 1)
            else:
                n.append(int(math.floor(q)) + 2)
        self.n_nodes = tuple(n)
        self.xmin = tuple(a for a, _ in self.lims)
        self.h_inv = 1.0 / self.h

    @property
    def dim(self) -> int:
        return len(self.n_nodes)

    def size(self) -> tuple:
        return self.n_nodes

    @property
    def nnodes(self) -> int:
        return int(np.prod(self.n_nodes))

    def nblocks(self) -> tuple:
        L = self.block_size_log2
        return tuple(((n - 1) >> L) + 1 for n in self.n_nodes)

    @property
    def nblocks_total(self) -> int:
        return int(np.prod(self.nblocks()))

    def spacing(self) -> float:
        return self.h

    def struct(self) -> _abi.tb_mesh:
        s = _abi.tb_mesh()
        s.dim = self.dim
        s.block_log2 = self.block_size_log2
        for d in range(3):
            s.n_nodes[d] = self.n_nodes[d] if d < self.dim else 1
            s.xmin[d] = self.xmin[d] if d < self.dim else 0.0
        s.h = self.h
        s.h_inv = self.h_inv
        return s

    def axis(self, d: int) -> np.ndarray:
        return self.xmin[d] + np.arange(self.n_nodes[d], dtype=np.float64) * self.h


# ---------------------------------------------------------------------------
# containers
# ---------------------------------------------------------------------------

def _alloc(backend, shape, dtype, device=None, fill=0.0):
    """numpy (host), pinned (page-locked host, returned as a numpy view) or torch (device)."""
    if backend == "numpy":
        a = np.empty(shape, dtype=dtype)
        a.fill(fill)
        return a
    import torch
    if backend == "pinned":
        tdt = {np.float64: torch.float64, np.float32: torch.float32, np.int32: torch.int32,
               np.int64: torch.int64}[np.dtype(dtype).type]
        a = torch.empty(shape, dtype=tdt, pin_memory=True).numpy()
        a.fill(fill)
        return a
    tdt = {np.float64: torch.float64, np.float32: torch.float32, np.int32: torch.int32,
           np.int64: torch.int64}[np.dtype(dtype).type]
    return torch.full(shape, fill, dtype=tdt, device=device)


def nsym(dim: int) -> int:
    return 6 if dim == 3 else 3


class Particles:
    """SoA particle state. Scalar type `dtype` (float64 or float32) for every
    field except F, which is float64 in both forms. With `x64=True` (float32
    only) the positions are float64 as well: the FP64-position form."""

    FIELDS = ("x", "v", "V", "m", "l", "grad_v", "sigma", "F", "B", "V0", "mu", "lam", "eps_p", "Cp_inv")
    OPTIONAL = ("m", "l", "B", "V0", "mu", "lam", "eps_p", "Cp_inv")

    def __init__(self, n, dim, dtype=np.float64, backend="numpy", device=None, optional=(), x64=False):
        self.n, self.dim, self.dtype = int(n), int(dim), np.dtype(dtype).type
        self.x64 = bool(x64) and self.dtype == np.float32
        self.backend, self.device = backend, device
        D = self.dim
        a = lambda shape, dt=self.dtype, fill=0.0: _alloc(backend, shape, dt, device, fill)  # noqa: E731
        self.x = a((D, self.n), np.float64 if self.x64 else self.dtype)
        self.v = a((D, self.n))
        self.V = a((self.n,))
        self.grad_v = a((D * D, self.n))
        self.sigma = a((nsym(D), self.n))
        self.F = a((D * D, self.n), np.float64)
        for k in range(D):
            self.F[k + k * D] = 1.0
        self.m = a((self.n,)) if "m" in optional else None
        self.l = a((self.n,)) if "l" in optional else None
        self.B = a((D * D, self.n)) if "B" in optional else None
        self.V0 = a((self.n,)) if "V0" in optional else None
        self.mu = a((self.n,)) if "mu" in optional else None
        self.lam = a((self.n,)) if "lam" in optional else None
        # von Mises plasticity state: equivalent plastic strain and the inverse
        # plastic right Cauchy-Green tensor (symmetric, identity at rest)
        self.eps_p = a((self.n,)) if "eps_p" in optional else None
        self.Cp_inv = a((nsym(D), self.n)) if "Cp_inv" in optional else None
        if self.Cp_inv is not None:
            for k in ((0, 3, 5) if D == 3 else (0, 2)):
                self.Cp_inv[k] = 1.0

    def __len__(self):
        return self.n

    def struct(self) -> _abi.tb_particles:
        s = _abi.tb_particles()
        D = self.dim
        s.n = self.n
        for d, p in enumerate(_row_ptrs(self.x, D)):
            s.x[d] = p
        for d, p in enumerate(_row_ptrs(self.v, D)):
            s.v[d] = p
        s.V = _ptr(self.V)
        s.m = _ptr(self.m)
        s.l = _ptr(self.l)
        for k, p in enumerate(_row_ptrs(self.grad_v, D * D)):
            s.grad_v[k] = p
        for k, p in enumerate(_row_ptrs(self.sigma, nsym(D))):
            s.sigma[k] = p
        for k, p in enumerate(_row_ptrs(self.F, D * D)):
            s.F[k] = p
        for k, p in enumerate(_row_ptrs(self.B, D * D)):
            s.B[k] = p
        s.V0 = _ptr(self.V0)
        s.mu = _ptr(self.mu)
        s.lambda_ = _ptr(self.lam)
        s.eps_p = _ptr(self.eps_p)
        for k, p in enumerate(_row_ptrs(self.Cp_inv, nsym(D))):
            s.Cp_inv[k] = p
        return s

    def to(self, backend, device=None, dtype=None, x64=None) -> "Particles":
        """Copy into another backend (numpy <-> torch) and/or scalar type
        (`x64`: float64 positions with a float32 state; default: as self)."""
        dtype = np.dtype(dtype or self.dtype).type
        x64 = self.x64 if x64 is None else bool(x64)
        opt = tuple(k for k in self.OPTIONAL if getattr(self, k) is not None)
        out = Particles(self.n, self.dim, dtype, backend, device, optional=opt, x64=x64)
        for k in self.FIELDS:
            src = getattr(self, k)
            if src is None:
                continue
            dst = getattr(out, k)
            srcn = src if isinstance(src, np.ndarray) else src.detach().cpu().numpy()
            tdt = np.float64 if (k == "F" or (k == "x" and out.x64)) else dtype
            if backend in ("numpy", "pinned"):
                dst[...] = srcn.astype(tdt)
            else:
                import torch
                dst.copy_(torch.from_numpy(np.ascontiguousarray(srcn.astype(tdt))))
        return out

    def numpy(self) -> dict:
        out = {}
        for k in self.FIELDS:
            a = getattr(self, k)
            if a is None:
                continue
            out[k] = a if isinstance(a, np.ndarray) else a.detach().cpu().numpy()
        return out


class Adjoint:
    """Sensitivities of a scalar loss to the particle state (x, v, F) and to the
    per-particle Lame parameters, all float64 in both precision forms (the
    tb_adjoint descriptor). `mu` / `lam` accumulate across steps."""

    def __init__(self, n, dim, backend="numpy", device=None, lame=True, apic=False):
        self.n, self.dim, self.backend = int(n), int(dim), backend
        D = self.dim
        a = lambda shape: _alloc(backend, shape, np.float64, device, 0.0)  # noqa: E731
        self.x = a((D, self.n))
        self.v = a((D, self.n))
        self.F = a((D * D, self.n))
        self.mu = a((self.n,)) if lame else None
        self.lam = a((self.n,)) if lame else None
        self.B = a((D * D, self.n)) if apic else None  # sensitivity to the APIC matrix

    def zero_(self):
        for k in ("x", "v", "F", "mu", "lam", "B"):
            arr = getattr(self, k)
            if arr is None:
                continue
            if isinstance(arr, np.ndarray):
                arr.fill(0.0)
            else:
                arr.zero_()
        return self

    def struct(self) -> _abi.tb_adjoint:
        s = _abi.tb_adjoint()
        D = self.dim
        for d, p in enumerate(_row_ptrs(self.x, D)):
            s.x[d] = p
        for d, p in enumerate(_row_ptrs(self.v, D)):
            s.v[d] = p
        for k, p in enumerate(_row_ptrs(self.F, D * D)):
            s.F[k] = p
        s.mu = _ptr(self.mu)
        s.lambda_ = _ptr(self.lam)
        for k, p in enumerate(_row_ptrs(self.B, D * D)):
            s.B[k] = p
        return s

    def numpy(self) -> dict:
        out = {}
        for k in ("x", "v", "F", "mu", "lam", "B"):
            a = getattr(self, k)
            if a is not None:
                out[k] = a if isinstance(a, np.ndarray) else a.detach().cpu().numpy()
        return out


class Grid:
    """SoA grid fields m, mv, f, v, vn over prod(n_nodes) column-major nodes.

    `sparse=True`: the block-sparse grid (`generate_grid(SpArray, ...)`,
    src/Grids/sparray.jl): the fields hold only the active node blocks
    (blocks of blockwidth^dim nodes, node block of node i = i >> block_size_log2
    per axis), `capacity` nodes each, in the storage order of the reference's
    SpIndices (storage block k - 1, then the column-major node inside the
    block); `block_numbering` (0 inactive, k >= 1), `active_blocks` (1-based
    node block ids in storage order) and `nactive` describe them, and
    runtime.update_sparsity fills them from particle positions."""

    def __init__(self, mesh: CartesianMesh, dtype=np.float64, backend="numpy", device=None, sparse=False,
                 capacity: int = 0):
        self.mesh, self.dtype, self.backend, self.device = mesh, np.dtype(dtype).type, backend, device
        self.sparse = bool(sparse)
        N, D = mesh.nnodes, mesh.dim
        if self.sparse:
            nb = mesh.nblocks_total
            ai = lambda k: _alloc(backend, (k,), np.int32, device, 0)  # noqa: E731
            self.block_numbering, self.active_blocks, self.nactive = ai(nb), ai(nb), ai(2)
            N = self._round_capacity(capacity)
        else:
            self.block_numbering = self.active_blocks = self.nactive = None
        self.capacity = N
        self._alloc_fields(N)

    @property
    def blocklength(self) -> int:
        return 1 << (self.mesh.block_size_log2 * self.mesh.dim)

    def _round_capacity(self, n: int) -> int:
        bl = self.blocklength
        return max(bl, -(-int(n) // bl) * bl)

    def _alloc_fields(self, N: int):
        D = self.mesh.dim
        a = lambda shape: _alloc(self.backend, shape, self.dtype, self.device)  # noqa: E731
        self.m = a((N,))
        self.mv = a((D, N))
        self.f = a((D, N))
        self.v = a((D, N))
        self.vn = a((D, N))

    def reserve(self, nodes: int):
        """Sparse grid: field arrays for at least `nodes` stored nodes (new,
        zeroed arrays when they grow)."""
        if not self.sparse:
            raise TypeError("reserve() is for a sparse grid")
        if nodes > self.capacity:
            self.capacity = self._round_capacity(nodes)
            self._alloc_fields(self.capacity)

    def struct(self) -> _abi.tb_grid:
        s = _abi.tb_grid()
        D = self.mesh.dim
        s.m = _ptr(self.m)
        for name in ("mv", "f", "v", "vn"):
            arr = getattr(s, name)
            for d, p in enumerate(_row_ptrs(getattr(self, name), D)):
                arr[d] = p
        if self.sparse:
            s.block_numbering = _ptr(self.block_numbering)
            s.active_blocks = _ptr(self.active_blocks)
            s.nactive = _ptr(self.nactive)
            s.capacity = self.capacity
        return s

    def numpy(self) -> dict:
        keys = ("m", "mv", "f", "v", "vn") + (("block_numbering", "active_blocks", "nactive") if self.sparse else ())
        return {k: (getattr(self, k) if isinstance(getattr(self, k), np.ndarray)
                    else getattr(self, k).detach().cpu().numpy()) for k in keys}

    def dense(self) -> dict:
        """The fields on every node (numpy), zeros where a sparse grid stores nothing."""
        g = self.numpy()
        if not self.sparse:
            return {k: g[k] for k in ("m", "mv", "f", "v", "vn")}
        mesh, D = self.mesh, self.mesh.dim
        n, nb, L = mesh.n_nodes, mesh.nblocks(), mesh.block_size_log2
        W = 1 << L
        k = int(g["nactive"][0])
        stored = np.arange(k * self.blocklength)
        blk = g["active_blocks"][stored >> (L * D)] - 1
        q = stored & (self.blocklength - 1)
        idx = []
        for d in range(D):
            b = (blk // int(np.prod(nb[:d]))) % nb[d]
            idx.append(b * W + (q // W ** d) % W)
        inside = np.all([idx[d] < n[d] for d in range(D)], axis=0)
        lin = np.zeros_like(stored)
        for d in reversed(range(D)):
            lin = lin * n[d] + idx[d]
        out = {}
        for key in ("m", "mv", "f", "v", "vn"):
            a = g[key]
            full = np.zeros(a.shape[:-1] + (mesh.nnodes,), dtype=a.dtype)
            full[..., lin[inside]] = a[..., stored[inside]]
            out[key] = full
        return out


class Partition:
    """GPUBlockStrategy arrays (src/Parallel/gpu_block_strategy.jl:10-22)."""

    def __init__(self, mesh: CartesianMesh, n: int, backend="numpy", device=None):
        nb = mesh.nblocks_total
        a = lambda k: _alloc(backend, (k,), np.int32, device, 0)  # noqa: E731
        self.mesh, self.nblocks = mesh, nb
        self.blockids = a(n)
        self.counts = a(nb)
        self.offsets = a(nb + 1)
        self.blocklist = a(nb)
        self.particleindices = a(n)
        self.nactive = 0
        self.nassigned = 0

    def struct(self) -> _abi.tb_partition:
        s = _abi.tb_partition()
        for k in ("blockids", "counts", "offsets", "blocklist", "particleindices"):
            setattr(s, k, _ptr(getattr(self, k)))
        s.nblocks = self.nblocks
        return s

    def numpy(self) -> dict:
        return {k: (getattr(self, k) if isinstance(getattr(self, k), np.ndarray)
                    else getattr(self, k).detach().cpu().numpy())
                for k in ("blockids", "counts", "offsets", "blocklist", "particleindices")}


class BasisWeights:
    """Stored BasisWeightArray layout (src/Basis/basis_weight.jl:345-358)."""

    def __init__(self, dim, n, dtype=np.float64, backend="numpy", device=None):
        nw = 3 ** dim
        self.dim, self.n = dim, n
        self.w = _alloc(backend, (n, nw), dtype, device)
        self.grad_w = _alloc(backend, (n, nw, dim), dtype, device)
        self.window = _alloc(backend, (n, 2 * dim), np.int64, device, 0)

    def struct(self) -> _abi.tb_weights:
        s = _abi.tb_weights()
        s.w, s.grad_w, s.window = _ptr(self.w), _ptr(self.grad_w), _ptr(self.window)
        return s


@dataclass(frozen=True)
class GridSampling:
    """GridSampling(spacing = 1/2) (src/particles.jl:3-11): particles aligned with
    the grid at `spacing * h`, so `spacing = 1/k` gives k^dim particles per cell."""

    spacing: float = 0.5


def sampling_axes(alg: GridSampling, mesh: CartesianMesh, box=None) -> list[np.ndarray]:
    """The per-axis coordinates of `alg`'s points over `mesh`: `(xmin + l/2):l:xmax`
    with `l = spacing * h` (src/particles.jl:13-18), each kept inside
    `box[d] = (lo, hi)` (lo <= x <= hi) when given."""
    if not isinstance(alg, GridSampling):
        raise TypeError("generate_points: only GridSampling is on the B200 path "
                        "(PoissonDiskSampling is the third-party PoissonDiskSampling.jl)")
    l = float(alg.spacing) * mesh.h
    axes = []
    for d in range(mesh.dim):
        xmin = mesh.xmin[d]
        xmax = mesh.xmin[d] + (mesh.n_nodes[d] - 1) * mesh.h
        # Julia's (xmin + l/2):l:xmax: the largest k with xmin + l/2 + k l <= xmax
        n = int(np.floor((xmax - (xmin + l / 2)) / l + 1e-9)) + 1
        ax = xmin + (2.0 * np.arange(n) + 1.0) * (l / 2.0)
        if box is not None and box[d] is not None:
            lo, hi = box[d]
            ax = ax[(ax >= lo) & (ax <= hi)]
        axes.append(ax)
    return axes


def generate_points(alg: GridSampling, mesh: CartesianMesh, box=None) -> np.ndarray:
    """The sample points of `alg` over `mesh` (src/particles.jl:13-18), shape
    (dim, n) in the reference's column-major order (first axis fastest). `box`
    (one (lo, hi) pair per axis, or None) keeps the points with lo <= x <= hi on
    every axis: the same points, in the same order, as filtering the whole
    lattice with that box, without forming it (the lattice of a 256^3 mesh at 2
    per cell per axis has 134 M points)."""
    grids = np.meshgrid(*sampling_axes(alg, mesh, box), indexing="ij")
    return np.stack([g.reshape(-1, order="F") for g in grids])


def generate_particles(mesh: CartesianMesh, alg: GridSampling = GridSampling(), dtype=np.float64,
                       optional=(), backend="numpy", device=None, x64=False, box=None) -> Particles:
    """generate_particles(ParticleProp, mesh; alg) (src/particles.jl:112-118): a
    zero-initialised particle state (F = I, Cp_inv = I) with one particle per
    sample point of `alg`, positions set from the points. The reference's
    default `alg` is PoissonDiskSampling, a third-party algorithm that is not
    on this path; GridSampling is the default here. `optional` names the
    optional fields to allocate (m, l, B, V0, mu, lam, eps_p, Cp_inv); `box` is
    the box filter of `generate_points`."""
    pts = generate_points(alg, mesh, box)
    P = Particles(pts.shape[1], mesh.dim, np.float64, optional=optional)
    P.x[...] = pts
    if backend == "numpy" and np.dtype(dtype) == np.float64 and not x64:
        return P
    return P.to(backend, device=device, dtype=dtype, x64=x64)


def generate_grid(mesh: CartesianMesh, dtype=np.float64, backend="numpy", device=None, sparse=False,
                  capacity: int = 0) -> Grid:
    """generate_grid(GridProp, mesh) (src/Grids/grid.jl); `sparse=True` is
    generate_grid(SpArray, GridProp, mesh) (src/Grids/sparray.jl)."""
    return Grid(mesh, dtype, backend, device, sparse, capacity)


def generate_basis_weights(dim, n, dtype=np.float64, backend="numpy", device=None) -> BasisWeights:
    return BasisWeights(dim, n, dtype, backend, device)


# ---------------------------------------------------------------------------
# step parameters
# ---------------------------------------------------------------------------

def lame(E: float, nu: float) -> tuple[float, float]:
    """(mu, lambda) from Young's modulus and Poisson's ratio (README.md:50)."""
    lam = (E * nu) / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    return mu, lam


def step_params(dt, mass=0.0, V0=0.0, mu=0.0, lam=0.0, gravity=(0.0, 0.0, 0.0), gimp_l=0.0,
                flip_alpha=1.0, basis=_abi.TB_BSPLINE_QUADRATIC, transfer=_abi.TB_TRANSFER_FLIP,
                material=_abi.MATERIAL_NEOHOOKEAN, wall_mask=0, wall_layers=0, hardening=0.0,
                yield_stress=0.0) -> _abi.tb_step_params:
    s = _abi.tb_step_params()
    s.dt, s.mass, s.V0, s.mu, s.lambda_ = dt, mass, V0, mu, lam
    for d in range(3):
        s.gravity[d] = gravity[d] if d < len(gravity) else 0.0
    s.gimp_l, s.flip_alpha = gimp_l, flip_alpha
    s.basis, s.transfer, s.material = basis, transfer, material
    s.wall_mask, s.wall_layers, s.reserved = wall_mask, wall_layers, 0
    s.hardening, s.yield_stress = hardening, yield_stress
    return s
