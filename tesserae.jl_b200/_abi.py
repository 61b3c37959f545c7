"""ctypes mirror of include/tesserae_b200.h and the loader of libtesserae_b200.so.

The structures here are byte-for-byte the POD descriptors of the C ABI. The
product library is loaded from this package's ``csrc/`` build folder; a missing
library is an error (there is no CPU fallback for the hot path).
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

TB_OK = 0
TB_ERR_ARG = -1
TB_ERR_CUDA = -2
TB_ERR_CAPACITY = -3
TB_ERR_UNSUPPORTED = -4
TB_ERR_DEVICE = -5

TB_BSPLINE_QUADRATIC = 0
TB_UGIMP = 1
TB_WLS_BSPLINE_QUADRATIC = 2
TB_WLS_UGIMP = 3
TB_KC_BSPLINE_QUADRATIC = 4
TB_KC_UGIMP = 5

TB_TRANSFER_FLIP = 0
TB_TRANSFER_APIC = 1

MATERIAL_NEOHOOKEAN = 0
MATERIAL_FLUID = 1
MATERIAL_VONMISES = 2

VP = C.c_void_p


class tb_mesh(C.Structure):
    _fields_ = [
        ("dim", C.c_int32),
        ("block_log2", C.c_int32),
        ("n_nodes", C.c_int64 * 3),
        ("xmin", C.c_double * 3),
        ("h", C.c_double),
        ("h_inv", C.c_double),
    ]


class tb_particles(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("x", VP * 3),
        ("v", VP * 3),
        ("V", VP),
        ("m", VP),
        ("l", VP),
        ("grad_v", VP * 9),
        ("sigma", VP * 6),
        ("F", VP * 9),
        ("B", VP * 9),
        ("V0", VP),
        ("mu", VP),
        ("lambda_", VP),
        ("eps_p", VP),
        ("Cp_inv", VP * 6),
    ]


class tb_grid(C.Structure):
    _fields_ = [("m", VP), ("mv", VP * 3), ("f", VP * 3), ("v", VP * 3), ("vn", VP * 3),
                ("block_numbering", VP), ("active_blocks", VP), ("nactive", VP), ("capacity", C.c_int64)]


class tb_partition(C.Structure):
    _fields_ = [
        ("blockids", VP),
        ("counts", VP),
        ("offsets", VP),
        ("blocklist", VP),
        ("particleindices", VP),
        ("nblocks", C.c_int64),
    ]


class tb_weights(C.Structure):
    _fields_ = [("w", VP), ("grad_w", VP), ("window", VP)]


class tb_step_params(C.Structure):
    _fields_ = [
        ("dt", C.c_double),
        ("mass", C.c_double),
        ("V0", C.c_double),
        ("mu", C.c_double),
        ("lambda_", C.c_double),
        ("gravity", C.c_double * 3),
        ("gimp_l", C.c_double),
        ("flip_alpha", C.c_double),
        ("basis", C.c_int32),
        ("transfer", C.c_int32),
        ("material", C.c_int32),
        ("wall_mask", C.c_int32),
        ("wall_layers", C.c_int32),
        ("reserved", C.c_int32),
        ("hardening", C.c_double),
        ("yield_stress", C.c_double),
    ]


class tb_adjoint(C.Structure):
    _fields_ = [("x", VP * 3), ("v", VP * 3), ("F", VP * 9), ("mu", VP), ("lambda_", VP), ("B", VP * 9)]


class tb_kernel_time(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_int64), ("ms", C.c_double)]


P = C.POINTER
I32 = C.c_int32
I64 = C.c_int64

# (name, restype, argtypes) of every symbol the header declares.
SIGNATURES = [
    ("tb_create", VP, [I32, VP]),
    ("tb_destroy", None, [VP]),
    ("tb_last_error", C.c_char_p, [VP]),
    ("tb_set_stream", I32, [VP, VP]),
    ("tb_synchronize", I32, [VP]),
    ("tb_launch_count", I64, [VP]),
    ("tb_profile_enable", I32, [VP, I32]),
    ("tb_profile_read", I32, [VP, P(tb_kernel_time), I32, P(I32)]),
    ("tb_bin_particles_noalloc", I32, [P(tb_mesh), P(tb_particles), I32, P(tb_partition), VP, P(I64), P(I64),
                                       C.c_char_p, I32]),
    ("tb_tape_bytes", I64, [P(tb_mesh), I64, I32, I32, I32, I32, I32]),
    ("tb_update_sparsity_f64", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid), P(I64)]),
    ("tb_update_sparsity_f32", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid), P(I64)]),
    ("tb_update_sparsity_f32x64", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid), P(I64)]),
    ("tb_tape_release", I32, [VP]),
]
for _p in ("f64", "f32"):
    SIGNATURES += [
        (f"tb_update_weights_{_p}", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_step_params), P(tb_weights)]),
        (f"tb_bin_particles_{_p}", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(I64), P(I64)]),
        (f"tb_p2g_{_p}", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid), P(tb_step_params)]),
        (f"tb_grid_update_{_p}", I32, [VP, P(tb_mesh), P(tb_grid), P(tb_step_params)]),
        (f"tb_g2p_{_p}", I32, [VP, P(tb_mesh), P(tb_grid), P(tb_particles), P(tb_step_params)]),
        (f"tb_step_{_p}", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid), P(tb_step_params), I32]),
        (f"tb_rollout_host_{_p}", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_step_params), I32]),
        (f"tb_adjoint_step_{_p}", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid),
                                        P(tb_step_params), P(tb_adjoint)]),
        (f"tb_tape_forward_{_p}", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid),
                                        P(tb_step_params), I32, I32]),
        (f"tb_tape_backward_{_p}", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid),
                                         P(tb_step_params), P(tb_adjoint)]),
    ]

SIGNATURES += [
    ("tb_step_f32x64", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid), P(tb_step_params), I32]),
    ("tb_adjoint_step_f32x64", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid),
                                     P(tb_step_params), P(tb_adjoint)]),
    ("tb_tape_forward_f32x64", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid),
                                     P(tb_step_params), I32, I32]),
    ("tb_tape_backward_f32x64", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid),
                                      P(tb_step_params), P(tb_adjoint)]),
    ("tb_rollout_host_f32x64", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_step_params), I32]),
    ("tb_particle_contiguity", I32, [VP, P(tb_partition), I64, P(C.c_double)]),
    ("tb_max_wave_speed_f64", I32, [VP, I32, P(tb_particles), P(tb_step_params), P(C.c_double)]),
    ("tb_g2p2g_f64", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid), P(tb_step_params)]),
    ("tb_g2p2g_f32", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid), P(tb_step_params)]),
    ("tb_g2p2g_f32x64", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid), P(tb_step_params)]),
    ("tb_max_wave_speed_f32", I32, [VP, I32, P(tb_particles), P(tb_step_params), P(C.c_double)]),
]
for _p in ("f64", "f32", "f32x64"):
    SIGNATURES += [
        (f"tb_reorder_particles_{_p}", I32, [VP, I32, P(tb_particles), P(tb_partition), C.c_double, P(I32)]),
        (f"tb_step_reorder_{_p}", I32, [VP, P(tb_mesh), P(tb_particles), P(tb_partition), P(tb_grid),
                                        P(tb_step_params), I32, C.c_double]),
    ]

PKG_DIR = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "csrc" / "libtesserae_b200.so"

_lib = None


def load_library(path: os.PathLike | None = None) -> C.CDLL:
    """Load libtesserae_b200.so and bind every declared symbol (raises if absent)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = pathlib.Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"libtesserae_b200.so not found at {p}; build it with "
            "`python __graft_entry__.py` or `make -C 'tesserae.jl_b200/csrc'`")
    lib = C.CDLL(str(p))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def declared_symbols() -> list[str]:
    return [s[0] for s in SIGNATURES]
