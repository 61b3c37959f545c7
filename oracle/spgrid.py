"""Block-sparse grid (SpGrid) numbering restated in numpy: the oracle of
tb_update_sparsity_* and of the sparse grid's storage order.

TEST INFRASTRUCTURE ONLY: imported by tests/. The product package never
imports this module.

  occupied blocks   src/Grids/sparsity.jl:120-139   findblock of every particle
                                                    inside the mesh
  active blocks     src/Grids/sparsity.jl:192-200   each occupied block with its
                                                    3^dim neighbourhood, clipped
  numbering         src/Grids/sparsity.jl:50-58     ascending linear block id:
                                                    k = 1, 2, ... ; 0 inactive
  storage index     src/Grids/spindices.jl:87-100   (k - 1) blocklength + the
                                                    node's column-major index
                                                    inside its block
"""
from __future__ import annotations

import numpy as np


def occupied_blocks(mesh, x) -> np.ndarray:
    """Boolean (column-major flat) array over nblocks(mesh): a block holds a
    particle inside the mesh (findblock, src/Mesh/cartesian.jl:277-285)."""
    L, nb = mesh.block_size_log2, mesh.nblocks()
    inside = np.ones(x.shape[1], dtype=bool)
    lin = np.zeros(x.shape[1], dtype=np.int64)
    for d in reversed(range(mesh.dim)):
        c = np.floor((x[d] - x.dtype.type(mesh.xmin[d])) * x.dtype.type(mesh.h_inv))
        inside &= (c >= 0) & (c <= mesh.n_nodes[d] - 2)
        lin = lin * nb[d] + (np.where(inside, c, 0).astype(np.int64) >> L)
    occ = np.zeros(mesh.nblocks_total, dtype=bool)
    occ[lin[inside]] = True
    return occ


def active_blocks(mesh, occupied: np.ndarray) -> np.ndarray:
    """Each occupied block and its neighbours within one block per axis."""
    nb = mesh.nblocks()
    occ = occupied.reshape(nb, order="F")
    act = np.zeros_like(occ)
    for off in np.ndindex(*([3] * mesh.dim)):
        src, dst = [], []
        for d, o in enumerate(off):
            o -= 1
            src.append(slice(max(0, -o), nb[d] - max(0, o)))
            dst.append(slice(max(0, o), nb[d] - max(0, -o)))
        act[tuple(dst)] |= occ[tuple(src)]
    return act.ravel(order="F")


def numbering(mesh, x):
    """(block_numbering int32, active_blocks int32 1-based ids in storage
    order, nactive) after update_sparsity!(grid, x)."""
    act = active_blocks(mesh, occupied_blocks(mesh, x))
    num = np.zeros(mesh.nblocks_total, dtype=np.int32)
    ids = np.flatnonzero(act)
    num[ids] = np.arange(1, ids.size + 1, dtype=np.int32)
    return num, (ids + 1).astype(np.int32), int(ids.size)


def storage_index(mesh, num: np.ndarray, node) -> int:
    """0-based storage slot of node (0-based indices), -1 if its block is inactive."""
    L, nb, W = mesh.block_size_log2, mesh.nblocks(), 1 << mesh.block_size_log2
    B, q, sb, sq = 0, 0, 1, 1
    for d in range(mesh.dim):
        B += (node[d] >> L) * sb
        q += (node[d] & (W - 1)) * sq
        sb *= nb[d]
        sq *= W
    k = int(num[B])
    return -1 if k == 0 else (k - 1) * W ** mesh.dim + q
