"""Seeded synthetic scenes for the five workloads of the explicit MPM path.

Every scene is generated on the host in FP64 with numpy's PCG64 generator from a
fixed seed, using the reference's GridSampling rule (src/particles.jl:9-16,
26-31: points at xmin + l/2 + k*l with l = spacing*h, kept in column-major
order, then filtered). No public dataset is involved.

Scenes:
  readme2d   2D two-disk collision of README.md:44-96 (100x100 cells, ~10k particles)
  cube3d     3D unit cube 256^3, centre cube of side 0.5, 2^3 per cell (16 777 216 particles)
  clusters3d 3D 512^3, 64 Gaussian clusters, lognormal masses (32M particles)
  sphere3d   3D 64^3 sphere r=0.3, jittered 4^3 per cell (the differentiable rollout)
  dambreak3d 3D 384^3 column [0,0.4]x[0,1]x[0,0.8], 2^3 per cell, WLS(uGIMP) + APIC fluid
  taylor3d   3D Taylor impact of docs/src/gpu.md:202-392: copper rod at 227 m/s onto a
             slip floor, KernelCorrection(BSpline(Quadratic())), von Mises plasticity,
             adaptive time step (~1.48M particles)
Each takes a `scale` that shrinks the mesh (cells per axis divided by `scale`,
spacing kept) so tests run the same physics at sizes the oracle finishes fast.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _abi
from .state import CartesianMesh, GridSampling, Particles, generate_points, lame, sampling_axes, step_params

SEEDS = {"readme2d": 0, "cube3d": 20260001, "clusters3d": 20260002, "sphere3d": 20260003,
         "dambreak3d": 20260004, "taylor3d": 20260005}


@dataclass
class Scene:
    name: str
    mesh: CartesianMesh
    particles: Particles          # host FP64
    params: _abi.tb_step_params
    nsteps: int
    meta: dict


def grid_sampling_axis(xmin: float, xmax: float, h: float, spacing: float = 0.5) -> np.ndarray:
    """Axis of GridSampling points: (xmin + l/2):l:xmax with l = spacing*h."""
    l = spacing * h
    n = int(np.floor((xmax - (xmin + l / 2)) / l + 1e-9)) + 1
    return xmin + (2.0 * np.arange(n) + 1.0) * (l / 2.0)


def _lattice(axes: list[np.ndarray]) -> np.ndarray:
    """Column-major (first axis fastest) lattice points, shape (dim, n)."""
    grids = np.meshgrid(*axes, indexing="ij")
    return np.stack([g.reshape(-1, order="F") for g in grids])


def readme2d(scale: int = 1) -> Scene:
    """README.md:44-96: unit square, h = 0.01, two disks r = 0.2, E = 500, nu = 0.3,
    rho0 = 1e3, dt = 1e-3; V0 = volume / N before the disk filter (README.md:57)."""
    h = 0.01
    L = 1.0 / scale
    mesh = CartesianMesh(h, (0.0, L), (0.0, L))
    pts = generate_points(GridSampling(), mesh)
    npre = pts.shape[1]
    V0 = (L * L) / npre
    rho0, E, nu = 1e3, 500.0, 0.3
    r = 0.2 * L
    keep = (np.hypot(pts[0] - r, pts[1] - r) < r) | (np.hypot(pts[0] - (L - r), pts[1] - (L - r)) < r)
    pts = pts[:, keep]
    n = pts.shape[1]
    P = Particles(n, 2, np.float64)
    P.x[...] = pts
    s = np.where(pts[0] > 0.5 * L, -0.1, 0.1)
    P.v[0] = s
    P.v[1] = s
    P.V[...] = V0
    mu, lam = lame(E, nu)
    prm = step_params(1e-3, mass=rho0 * V0, V0=V0, mu=mu, lam=lam)
    return Scene("readme2d", mesh, P, prm, 1000, {"n_before_filter": npre, "E": E, "nu": nu, "rho0": rho0})


def cube3d(scale: int = 1, seed: int | None = None) -> Scene:
    """Unit cube 256^3 cells (h = 1/256), centre cube [1/4, 3/4]^3 at 2 particles
    per cell per axis, v ~ U[-0.5, 0.5]^3, Neo-Hookean E = 1e6, nu = 0.3,
    rho0 = 1e3, gravity -9.81 z, 100 steps. The stated dt = 1e-4 puts the P-wave
    CFL number c dt / h at 0.94 (c = sqrt((lambda + 2 mu) / rho0) = 36.7 m/s), and the
    FP64 oracle goes to NaN within 20 steps; dt = 5e-5 (CFL 0.47) is used instead."""
    cells = 256 // scale
    h = 1.0 / 256
    L = cells * h
    mesh = CartesianMesh(h, (0.0, L), (0.0, L), (0.0, L))
    lpart = h / 2
    # GridSampling over the mesh, kept inside the centre cube [L/4, 3L/4]^3
    pts = generate_points(GridSampling(), mesh, box=[(L / 4, 3 * L / 4)] * 3)
    n = pts.shape[1]
    rng = np.random.default_rng(SEEDS["cube3d"] if seed is None else seed)
    P = Particles(n, 3, np.float64)
    P.x[...] = pts
    P.v[...] = rng.uniform(-0.5, 0.5, size=(3, n))
    V0 = lpart ** 3
    P.V[...] = V0
    rho0, E, nu = 1e3, 1e6, 0.3
    mu, lam = lame(E, nu)
    prm = step_params(5e-5, mass=rho0 * V0, V0=V0, mu=mu, lam=lam, gravity=(0.0, 0.0, -9.81))
    return Scene("cube3d", mesh, P, prm, 100, {"E": E, "nu": nu, "rho0": rho0, "cells": cells})


def _lattice_on_device(mesh: CartesianMesh, box, device, dtype, optional=(), x64=False) -> Particles:
    """Particles on `device` (torch) at the GridSampling points of `mesh` inside
    `box`, in the column-major order of `generate_points`, built from the axes
    on the device without forming the points on the host."""
    import torch
    axes = sampling_axes(GridSampling(), mesh, box)
    sizes = [len(a) for a in axes]
    n = int(np.prod(sizes))
    P = Particles(n, mesh.dim, dtype, backend="torch", device=device, optional=optional, x64=x64)
    stride = 1
    for d in range(mesh.dim):
        a = torch.from_numpy(axes[d]).to(device=device, dtype=P.x.dtype)
        P.x[d].copy_(a.repeat_interleave(stride).repeat(n // (stride * sizes[d])))
        stride *= sizes[d]
    return P


def _sort_by_block(mesh: CartesianMesh, pts: np.ndarray) -> np.ndarray:
    """Stable order by reference block id: the particle order `reorder_particles!`
    establishes (src/Parallel/gpu_block_strategy.jl:173-238)."""
    L = mesh.block_size_log2
    nb = mesh.nblocks()
    b = np.zeros(pts.shape[1], dtype=np.int64)
    for d in reversed(range(mesh.dim)):
        c = np.floor((pts[d] - mesh.xmin[d]) * mesh.h_inv).astype(np.int64) >> L
        b = b * nb[d] + np.clip(c, 0, nb[d] - 1)
    return np.argsort(b, kind="stable")


def block_ordered(scene: Scene) -> Scene:
    """`scene` with its particles stored in block order, in place: the order
    `reorder_particles!(particles, partition)` leaves them in after the first
    `update!(partition, particles.x)`, the set-up docs/src/parallel.md:47-57
    gives for GPU runs. Every particle field is permuted alike; the particles
    themselves are unchanged."""
    P = scene.particles
    order = _sort_by_block(scene.mesh, P.x)
    for k in Particles.FIELDS:
        a = getattr(P, k)
        if a is not None:
            a[...] = a[..., order]
    scene.meta["particle_order"] = "block"
    return scene


def clusters3d(scale: int = 1, n_total: int = 32 * 1024 * 1024, seed: int | None = None) -> Scene:
    """512^3 cells (h = 1/512), n_total particles from 64 Gaussian clusters
    (sigma = 0.02, centres U[0.2, 0.8]^3), masses rho0 V0 lognormal(0, 0.5),
    Neo-Hookean E = 1e5, nu = 0.35, 50 steps at dt = 2.5e-5. Points outside
    [0.01, 0.99]^3 of the (scaled) domain are redrawn. Particles are stored
    block-ordered. dt: at the configuration's 5e-5 the scene is unstable (up to
    ~31 overlapping particles per cell and light lognormal masses put the local
    CFL number above 1): an FP64 run whose velocities are perturbed by 1e-7 is
    NaN within 30 steps; only the exactly uniform free fall of the unperturbed
    FP64 run survives. Every form is stable at 2.5e-5."""
    cells = 512 // scale
    h = 1.0 / 512
    L = cells * h
    mesh = CartesianMesh(h, (0.0, L), (0.0, L), (0.0, L))
    rng = np.random.default_rng(SEEDS["clusters3d"] if seed is None else seed)
    n = n_total // (scale ** 3)
    centres = rng.uniform(0.2 * L, 0.8 * L, size=(64, 3))
    which = rng.integers(0, 64, size=n)
    sig = 0.02 * L
    pts = centres[which].T + rng.normal(0.0, sig, size=(3, n))
    redrawn = 0
    while True:
        bad = np.any((pts < 0.01 * L) | (pts > 0.99 * L), axis=0)
        nbad = int(bad.sum())
        if nbad == 0:
            break
        redrawn += nbad
        pts[:, bad] = centres[which[bad]].T + rng.normal(0.0, sig, size=(3, nbad))
    order = _sort_by_block(mesh, pts)
    pts = pts[:, order]
    P = Particles(n, 3, np.float64, optional=("m",))
    P.x[...] = pts
    V0 = (h / 2) ** 3
    rho0, E, nu = 1e3, 1e5, 0.35
    P.m[...] = rho0 * V0 * rng.lognormal(0.0, 0.5, size=n)
    P.V[...] = V0
    mu, lam = lame(E, nu)
    prm = step_params(2.5e-5, mass=rho0 * V0, V0=V0, mu=mu, lam=lam, gravity=(0.0, 0.0, -9.81))
    return Scene("clusters3d", mesh, P, prm, 50, {"E": E, "nu": nu, "rho0": rho0, "redrawn": redrawn})


def sphere3d(scale: int = 1, seed: int | None = None) -> Scene:
    """64^3 cells (h = 1/64), sphere r = 0.3 at (0.5, 0.5, 0.5), 4 particles per cell
    per axis on a lattice jittered by U[-l/4, l/4], per-particle log E = log(1e5) +
    N(0, 0.1), nu = 0.3, rho0 = 1e3, dt = 5e-4, 200 steps. The initial velocity is
    not part of the configuration; it is set to (0, 0, 0.5) + U[-0.1, 0.1]^3 per
    particle, so the sphere moves toward the loss target (0.5, 0.5, 0.8) and deforms."""
    cells = 64 // scale
    h = 1.0 / 64
    L = cells * h
    mesh = CartesianMesh(h, (0.0, L), (0.0, L), (0.0, L))
    rng = np.random.default_rng(SEEDS["sphere3d"] if seed is None else seed)
    pts = generate_points(GridSampling(0.25), mesh)
    c, r = 0.5 * L, 0.3 * L
    keep = np.sum((pts - c) ** 2, axis=0) < r * r
    pts = pts[:, keep]
    lp = h / 4
    pts = pts + rng.uniform(-lp / 4, lp / 4, size=pts.shape)
    n = pts.shape[1]
    P = Particles(n, 3, np.float64, optional=("mu", "lam"))
    P.x[...] = pts
    V0 = lp ** 3
    P.V[...] = V0
    logE = np.log(1e5) + rng.normal(0.0, 0.1, size=n)
    P.v[...] = rng.uniform(-0.1, 0.1, size=(3, n))
    P.v[2] += 0.5
    mu, lam = lame(np.exp(logE), 0.3)
    P.mu[...] = mu
    P.lam[...] = lam
    prm = step_params(5e-4, mass=1e3 * V0, V0=V0, mu=float(np.mean(mu)), lam=float(np.mean(lam)))
    return Scene("sphere3d", mesh, P, prm, 200, {"nu": 0.3, "rho0": 1e3, "target": (0.5 * L, 0.5 * L, 0.8 * L)})


def dambreak3d(scale: int = 1, device=None, dtype=np.float64, x64: bool = False, particles: bool = True) -> Scene:
    """384^3 cells (h = 1/384), column [0,0.4]x[0,1]x[0,0.8] at 2^3 per cell,
    weakly compressible fluid p = -K (J - 1) with K = 2e6, rho0 = 1e3, WLS(uGIMP)
    basis with l = h/2, APIC transfer, slip walls on every face, 100 steps at
    dt = 2.5e-5. dt: the configuration's 5e-5 puts the acoustic CFL number
    (sqrt(K / rho0) dt / h) at 0.86; the FP32 run diverges within 50 steps and
    the FP64 run only survives unperturbed. Both are stable at 2.5e-5 (CFL 0.43).
    With `device`, the particles are built there directly in `dtype` (FP64
    positions with `x64`; the full
    scene has 145 M particles: 46 GB of FP64 host state otherwise); the state
    is deterministic (a lattice at rest), so both builds are the same scene."""
    cells = 384 // scale
    h = 1.0 / 384
    L = cells * h
    mesh = CartesianMesh(h, (0.0, L), (0.0, L), (0.0, L))
    box = [(0.0, 0.4 * L), None, (0.0, 0.8 * L)]
    V0 = (h / 2) ** 3
    if not particles:  # mesh and parameters only; the state is built per precision form
        P = None
    elif device is None:
        pts = generate_points(GridSampling(), mesh, box=box)
        n = pts.shape[1]
        P = Particles(n, 3, np.float64, optional=("B",))
        P.x[...] = pts
    else:
        P = _lattice_on_device(mesh, box, device, dtype, optional=("B",), x64=x64)
    if P is not None:
        P.V[...] = V0
    K = 2e6
    prm = step_params(2.5e-5, mass=1e3 * V0, V0=V0, mu=0.0, lam=K, gravity=(0.0, 0.0, -9.81),
                      gimp_l=h / 2, basis=_abi.TB_WLS_UGIMP, transfer=_abi.TB_TRANSFER_APIC,
                      material=_abi.MATERIAL_FLUID, wall_mask=0b111111, wall_layers=2)
    return Scene("dambreak3d", mesh, P, prm, 100, {"K": K, "rho0": 1e3, "scale": scale,
                                                   "built_on_device": device is not None or not particles})


SCENES = {"readme2d": readme2d, "cube3d": cube3d, "clusters3d": clusters3d, "sphere3d": sphere3d,
          "dambreak3d": dambreak3d}


def taylor3d(scale: int = 1, seed: int | None = None) -> Scene:
    """The Taylor impact of docs/src/gpu.md:202-392: rod R = 3.2 mm, L = 32.4 mm
    at (0, 0, -227) m/s onto a slip floor (the node layer z = 0 keeps no normal
    velocity), mesh spacing R/12 over (-3R, 3R)^2 x (0, 1.1 L) (the upper bound
    expanded to whole cells as CartesianMesh does), E = 117 GPa, nu = 0.35,
    rho0 = 8.93e3, von Mises with H = 0.1 GPa and tau_y0 = 0.4 GPa,
    KernelCorrection(BSpline(Quadratic())) weights, FLIP transfer, CFL 0.8 on
    c = sqrt((lambda + 2 mu) / rho) + |v|, up to t = 80 us (about 1.8k steps).
    Particles: the reference samples the rod's block of grid nodes with
    PoissonDiskSampling(spacing = 1/3) (a third-party algorithm not in the
    reference tree); the stand-in is a lattice of the same spacing (3 per cell
    per axis) jittered by U[-l/4, l/4], which gives the same count (1.48 M after
    the cylinder filter). V = block volume / particles before the filter, as the
    reference sets it. `scale` multiplies the spacing (same rod, 1/scale^3 of the
    particles)."""
    R, L = 0.0032, 0.0324
    h = R / 12 * scale
    mesh = CartesianMesh(h, (-3 * R, 3 * R), (-3 * R, 3 * R), (0.0, L + 0.1 * L))
    rng = np.random.default_rng(SEEDS["taylor3d"] if seed is None else seed)
    # extract(grid.x, (-R,R), (-R,R), (0,L)): the nodes inside the box
    zmax = np.floor(L / h + 1e-9) * h
    l = h / 3
    axx = grid_sampling_axis(-R, R, h, spacing=1 / 3)
    axz = grid_sampling_axis(0.0, zmax, h, spacing=1 / 3)
    pts = _lattice([axx, axx, axz])
    npre = pts.shape[1]
    Vp = (2 * R) * (2 * R) * zmax / npre
    pts = pts + rng.uniform(-l / 4, l / 4, size=pts.shape)
    pts = pts[:, pts[0] ** 2 + pts[1] ** 2 < R * R]
    n = pts.shape[1]
    P = Particles(n, 3, np.float64, optional=("eps_p", "Cp_inv"))
    P.x[...] = pts
    P.V[...] = Vp
    P.v[2] = -227.0
    E, nu, rho0 = 117e9, 0.35, 8.93e3
    mu, lam = lame(E, nu)
    prm = step_params(0.0, mass=rho0 * Vp, V0=Vp, mu=mu, lam=lam, basis=_abi.TB_KC_BSPLINE_QUADRATIC,
                      material=_abi.MATERIAL_VONMISES, wall_mask=1 << 4, wall_layers=1,
                      hardening=0.1e9, yield_stress=0.4e9)
    prm.dt = taylor_dt(P.v, P.V, prm.mass, mu, lam, h)
    return Scene("taylor3d", mesh, P, prm, 1805, {"E": E, "nu": nu, "rho0": rho0, "CFL": 0.8,
                                                 "t_stop": 80e-6, "n_before_filter": npre})


def taylor_dt(v, V, mass, mu, lam, h, cfl=0.8) -> float:
    """The Taylor impact's time step (docs/src/gpu.md:283-284): CFL h / max c with
    c = sqrt((lambda + 2 mu) / (m / V)) + |v| over the particles (host arrays)."""
    c = np.sqrt((lam + 2 * mu) / (mass / np.asarray(V, dtype=np.float64))) + np.linalg.norm(
        np.asarray(v, dtype=np.float64), axis=0)
    return float(cfl * h / np.max(c))

