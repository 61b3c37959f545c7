"""ctypes wrapper of the CPU oracle libtb_oracle.so.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py. The product package never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "libtb_oracle.so"

_lib = None


def build(force: bool = False) -> pathlib.Path:
    """Compile the oracle with its Makefile (g++ -fopenmp)."""
    if force or not LIB.exists() or LIB.stat().st_mtime < max(
            (HERE / f).stat().st_mtime for f in ("tb_oracle.cpp", "tb_oracle.hpp")):
        subprocess.run(["make", "-C", str(HERE), "-B" if force else "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return LIB


def lib(abi):
    """Load the oracle, binding signatures against the ABI structs of `abi`."""
    global _lib
    if _lib is not None:
        return _lib
    build()
    L = C.CDLL(str(LIB))
    P = C.POINTER
    i32, i64, dbl = C.c_int32, C.c_int64, C.c_double
    sigs = {
        "tbo_bin": [C.c_int, P(abi.tb_mesh), P(abi.tb_particles), P(abi.tb_partition), P(i64), P(i64)],
        "tbo_update_weights": [C.c_int, P(abi.tb_mesh), P(abi.tb_particles), P(abi.tb_step_params),
                               P(abi.tb_weights)],
        "tbo_p2g": [C.c_int, P(abi.tb_mesh), P(abi.tb_particles), P(abi.tb_grid), P(abi.tb_step_params)],
        "tbo_grid_update": [C.c_int, P(abi.tb_mesh), P(abi.tb_grid), P(abi.tb_step_params)],
        "tbo_g2p": [C.c_int, P(abi.tb_mesh), P(abi.tb_grid), P(abi.tb_particles), P(abi.tb_step_params)],
        "tbo_g2p2g": [C.c_int, P(abi.tb_mesh), P(abi.tb_particles), P(abi.tb_grid), P(abi.tb_step_params)],
        "tbo_step": [C.c_int, P(abi.tb_mesh), P(abi.tb_particles), P(abi.tb_grid), P(abi.tb_step_params),
                     C.c_int],
        "tbo_step_parallel": [C.c_int, P(abi.tb_mesh), P(abi.tb_particles), P(abi.tb_grid),
                              P(abi.tb_step_params), C.c_int, C.c_int, P(dbl)],
        "tbo_supportnodes": [C.c_int, P(abi.tb_mesh), C.c_int, P(dbl), dbl, P(i64)],
        "tbo_adjoint_step": [C.c_int, P(abi.tb_mesh), P(abi.tb_particles), P(abi.tb_grid),
                             P(abi.tb_step_params), P(abi.tb_adjoint)],
        "tbo_step_dual": [P(abi.tb_mesh), P(abi.tb_particles), P(abi.tb_grid), P(abi.tb_step_params), C.c_int],
    }
    for name, args in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.tbo_max_threads.restype = C.c_int
    L.tbo_max_threads.argtypes = []
    L.tbo_jet_bspline_quadratic.argtypes = [dbl, P(dbl), P(dbl)]
    L.tbo_jet_bspline_quadratic.restype = None
    L.tbo_jet_ugimp.argtypes = [dbl, dbl, P(dbl), P(dbl)]
    L.tbo_jet_ugimp.restype = None
    _lib = L
    return L


def _prec(dtype) -> int:
    import numpy as np
    return 0 if np.dtype(dtype) == np.float64 else 1


def _check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed with status {rc}")


class Oracle:
    """Convenience calls on host (numpy) state containers."""

    def __init__(self, abi):
        self.abi = abi
        self.L = lib(abi)

    def bin(self, mesh, particles, partition):
        na, nass = C.c_int64(), C.c_int64()
        ps, qs = particles.struct(), partition.struct()
        _check(self.L.tbo_bin(_prec(particles.dtype), C.byref(mesh.struct()), C.byref(ps), C.byref(qs),
                              C.byref(na), C.byref(nass)), "bin")
        partition.nactive, partition.nassigned = na.value, nass.value
        return na.value, nass.value

    def update_weights(self, mesh, particles, params, weights):
        _check(self.L.tbo_update_weights(_prec(particles.dtype), C.byref(mesh.struct()),
                                         C.byref(particles.struct()), C.byref(params),
                                         C.byref(weights.struct())), "update_weights")

    def p2g(self, mesh, particles, grid, params):
        _check(self.L.tbo_p2g(_prec(particles.dtype), C.byref(mesh.struct()), C.byref(particles.struct()),
                              C.byref(grid.struct()), C.byref(params)), "p2g")

    def grid_update(self, mesh, grid, params):
        _check(self.L.tbo_grid_update(_prec(grid.dtype), C.byref(mesh.struct()), C.byref(grid.struct()),
                                      C.byref(params)), "grid_update")

    def g2p(self, mesh, grid, particles, params):
        _check(self.L.tbo_g2p(_prec(particles.dtype), C.byref(mesh.struct()), C.byref(grid.struct()),
                              C.byref(particles.struct()), C.byref(params)), "g2p")

    def g2p2g(self, mesh, particles, grid, params):
        _check(self.L.tbo_g2p2g(_prec(particles.dtype), C.byref(mesh.struct()), C.byref(particles.struct()),
                                C.byref(grid.struct()), C.byref(params)), "g2p2g")

    def step(self, mesh, particles, grid, params, nsteps=1):
        _check(self.L.tbo_step(_prec(particles.dtype), C.byref(mesh.struct()), C.byref(particles.struct()),
                               C.byref(grid.struct()), C.byref(params), nsteps), "step")

    def step_parallel(self, mesh, particles, grid, params, nsteps=1, nthreads=0):
        phases = (C.c_double * 4)()
        _check(self.L.tbo_step_parallel(_prec(particles.dtype), C.byref(mesh.struct()),
                                        C.byref(particles.struct()), C.byref(grid.struct()), C.byref(params),
                                        nsteps, nthreads, phases), "step_parallel")
        return list(phases)

    def adjoint_step(self, mesh, particles, grid, params, adjoint):
        """One step backwards: `particles` is the start-of-step state, `adjoint`
        (an Adjoint on the numpy backend) is updated in place."""
        _check(self.L.tbo_adjoint_step(_prec(particles.dtype), C.byref(mesh.struct()),
                                       C.byref(particles.struct()), C.byref(grid.struct()), C.byref(params),
                                       C.byref(adjoint.struct())), "adjoint_step")

    def directional_derivative(self, mesh, particles, params, nsteps, seed: dict, outputs=("x", "v")):
        """Forward-mode derivative of `nsteps` sequential FP64 steps: the state
        of host FP64 `particles` is advanced in dual numbers whose derivative
        parts start as `seed` (field name -> array shaped like the field, zero
        for the fields not named); returns ({field: final value}, {field:
        derivative of the final value}) for `outputs`. `particles` is left
        unchanged."""
        import numpy as np
        from types import SimpleNamespace
        abi = self.abi
        fields = [k for k in particles.FIELDS if getattr(particles, k) is not None]
        duals = {}
        for k in fields:
            a = np.asarray(getattr(particles, k), dtype=np.float64)
            d = np.zeros(a.shape + (2,))
            d[..., 0] = a
            if k in seed:
                d[..., 1] = np.asarray(seed[k], dtype=np.float64)
            duals[k] = d

        def rows(a, k):
            return [a[i].ctypes.data for i in range(k)] if a.ndim == 3 else [a.ctypes.data]

        s = abi.tb_particles()
        D = particles.dim
        s.n = particles.n
        nsym = 6 if D == 3 else 3
        for name, k, cnt in (("x", "x", D), ("v", "v", D), ("grad_v", "grad_v", D * D), ("sigma", "sigma", nsym),
                             ("F", "F", D * D), ("B", "B", D * D), ("Cp_inv", "Cp_inv", nsym)):
            if k in duals:
                for i, ptr in enumerate(rows(duals[k], cnt)):
                    getattr(s, name)[i] = ptr
        for name, k in (("V", "V"), ("m", "m"), ("l", "l"), ("V0", "V0"), ("mu", "mu"), ("lambda_", "lam"),
                        ("eps_p", "eps_p")):
            if k in duals:
                setattr(s, name, duals[k].ctypes.data)
        nn = mesh.nnodes
        gd = {k: np.zeros((D, nn, 2)) for k in ("mv", "f", "v", "vn")}
        gm = np.zeros((nn, 2))
        g = abi.tb_grid()
        g.m = gm.ctypes.data
        for k, arr in gd.items():
            for i in range(D):
                getattr(g, k)[i] = arr[i].ctypes.data
        _check(self.L.tbo_step_dual(C.byref(mesh.struct()), C.byref(s), C.byref(g), C.byref(params), nsteps),
               "step_dual")
        return ({k: duals[k][..., 0].copy() for k in outputs}, {k: duals[k][..., 1].copy() for k in outputs})

    def supportnodes(self, mesh, basis, x, l=0.0):
        xs = (C.c_double * 3)(*list(x) + [0.0] * (3 - len(x)))
        out = (C.c_int64 * 6)()
        _check(self.L.tbo_supportnodes(0, C.byref(mesh.struct()), basis, xs, l, out), "supportnodes")
        return [(out[2 * d], out[2 * d + 1]) for d in range(mesh.dim)]

    def jet_bspline_quadratic(self, xi):
        v, d = C.c_double(), C.c_double()
        self.L.tbo_jet_bspline_quadratic(xi, C.byref(v), C.byref(d))
        return v.value, d.value

    def jet_ugimp(self, xi, l):
        v, d = C.c_double(), C.c_double()
        self.L.tbo_jet_ugimp(xi, l, C.byref(v), C.byref(d))
        return v.value, d.value

    def max_threads(self):
        return self.L.tbo_max_threads()


def cores() -> int:
    return len(os.sched_getaffinity(0))
