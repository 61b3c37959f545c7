"""Shared comparison helpers for the parity tests."""
import numpy as np


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def max_rel(a, b, floor):
    """max |a - b| / max(|b|, floor)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


def basis_kind(abi, name):
    return {"bspline_quadratic": abi.TB_BSPLINE_QUADRATIC, "ugimp": abi.TB_UGIMP,
            "wls_bspline_quadratic": abi.TB_WLS_BSPLINE_QUADRATIC, "wls_ugimp": abi.TB_WLS_UGIMP,
            "kc_bspline_quadratic": abi.TB_KC_BSPLINE_QUADRATIC, "kc_ugimp": abi.TB_KC_UGIMP}[name]


def reference_partition(mesh, x):
    """Per-block particle lists by direct findblock, ascending particle order
    (test/partition.jl:80-93), as (blockids, counts, offsets, blocklist, perm)."""
    n = x.shape[1]
    L = mesh.block_size_log2
    nb = mesh.nblocks()
    inside = np.ones(n, dtype=bool)
    lin = np.zeros(n, dtype=np.int64)
    for d in reversed(range(mesh.dim)):
        c = np.floor((x[d] - x.dtype.type(mesh.xmin[d])) * x.dtype.type(mesh.h_inv))
        inside &= (c >= 0) & (c <= mesh.n_nodes[d] - 2)
        ci = np.where(inside, c, 0).astype(np.int64)
        lin = lin * nb[d] + (ci >> L)
    bid = np.where(inside, lin + 1, 0).astype(np.int32)
    counts = np.bincount(bid[bid > 0] - 1, minlength=mesh.nblocks_total).astype(np.int32)
    offsets = np.zeros(mesh.nblocks_total + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(counts)
    order = np.lexsort((np.arange(n), bid))
    perm = (order[bid[order] > 0] + 1).astype(np.int32)
    blocklist = (np.nonzero(counts)[0] + 1).astype(np.int32)
    return bid, counts, offsets.astype(np.int32), blocklist, perm
