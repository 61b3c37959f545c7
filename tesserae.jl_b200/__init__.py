"""tesserae_b200 -- B200-native (sm_100a) explicit MPM step of Tesserae.jl.

The package is the host side of libtesserae_b200.so: a mirror of the reference's
surface for the explicit MPM hot path (mesh, grid and particle containers, basis
weights, the block partition and the recognised @P2G / @G2P equation sets) that
calls the CUDA kernels through the C ABI declared in include/tesserae_b200.h.
"""
from . import _abi
from .state import (Adjoint, BasisWeights, CartesianMesh, Grid, GridSampling, Particles, Partition,
                    generate_basis_weights, generate_grid, generate_particles, generate_points, lame, step_params)
from . import export, scenes

__all__ = ["_abi", "Adjoint", "BasisWeights", "CartesianMesh", "Grid", "GridSampling", "Particles", "Partition",
           "generate_basis_weights", "generate_grid", "generate_particles", "generate_points", "lame", "step_params",
           "scenes", "export"]


def __getattr__(name):
    # The device API needs torch and the built library; import it lazily so the
    # host-only parts (scenes, containers) load without either.
    if name in ("runtime", "Context", "update", "P2G", "G2P", "step", "rollout_host", "adjoint_step",
                "tape_forward", "tape_backward", "rollout_grad", "RolloutFunction", "reorder_particles",
                "block_ordered_particle_contiguity"):
        import importlib
        runtime = importlib.import_module(__name__ + ".runtime")
        return runtime if name == "runtime" else getattr(runtime, name)
    raise AttributeError(name)
