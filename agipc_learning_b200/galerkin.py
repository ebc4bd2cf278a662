"""The AGIPC coarse space on the GPU (StiffGIPC/agipc/agipc_galerkin.cu).

A `GalerkinMapping` describes the mixed prolongation P of the reference's
coarse mapping (agipc_criterion.cuh:13-25): the first `prefix_blocks` fine
blocks pass through; FEM node k (fine block prefix_blocks + k) belongs to
coarse node fine_to_coarse[k], whose blocks start at prefix_blocks +
coarse_block_bases[c] and whose basis is the subset basis_masks[c] of
(1, x, y, z) at the node's rest position (1: translational, 15: affine).

`coarse_matrix`, `restrict` and `prolong` run A_c = P^T A P, b_c = P^T b and
x = P x_c through the C ABI; `coarse_solve` chains them with a MAS32 + PCG
solve of the coarse system on the same engine, prepared the way
replay_coarse_snapshot prepares one (identity partition, padding to a
multiple of 32 blocks; agipc_coarse_replay.cu:215-310).  The coarse solve
stops on ||b_c - A_c x_c|| <= tolerance ||b_c||; the reference's shadow solve
measures the residual against the fine right-hand side norm instead
(agipc_galerkin.cu:680-690).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .solver import MasPcg


@dataclass
class GalerkinMapping:
    prefix_blocks: int
    fine_to_coarse: np.ndarray      # int32 [fem_nodes]
    coarse_block_bases: np.ndarray  # int32 [coarse_nodes]
    basis_masks: np.ndarray         # int32 [coarse_nodes], 1..15
    rest_positions: np.ndarray      # float64 [fem_nodes, 3]
    coarse_block_nodes: int

    @property
    def fem_nodes(self) -> int:
        return int(len(self.fine_to_coarse))

    @property
    def fine_blocks(self) -> int:
        return self.prefix_blocks + self.fem_nodes

    @property
    def coarse_blocks(self) -> int:
        return self.prefix_blocks + self.coarse_block_nodes

    def _struct(self):
        keep = [np.ascontiguousarray(self.fine_to_coarse, np.int32),
                np.ascontiguousarray(self.coarse_block_bases, np.int32),
                np.ascontiguousarray(self.basis_masks, np.int32),
                np.ascontiguousarray(self.rest_positions, np.float64).reshape(-1)]
        ptr = [a.ctypes.data_as(ctypes.c_void_p) for a in keep]
        g = N.GalerkinMap(ptr[0], ptr[1], ptr[2], ptr[3], int(self.prefix_blocks), self.fem_nodes,
                          int(len(self.coarse_block_bases)), int(self.coarse_block_nodes))
        return g, keep


def coarse_matrix(m: MasPcg, mapping: GalerkinMapping, rows, cols, values9):
    """A_c = P^T A P from upper fine triplets (maspcg_galerkin_coarse_matrix):
    unique upper coarse blocks (rows, cols, values9 column-major)."""
    g, keep = mapping._struct()
    r = np.ascontiguousarray(rows, np.int32)
    c = np.ascontiguousarray(cols, np.int32)
    v = np.ascontiguousarray(values9, np.float64).reshape(-1, 9)
    cap = max(16 * len(r), 1)
    orow, ocol, oval = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros((cap, 9))
    n = ctypes.c_int()
    m._ck(m.lib.maspcg_galerkin_coarse_matrix(m.h, ctypes.byref(g), v.ctypes.data_as(ctypes.c_void_p),
                                              r.ctypes.data_as(ctypes.c_void_p), c.ctypes.data_as(ctypes.c_void_p),
                                              len(r), oval.ctypes.data_as(ctypes.c_void_p),
                                              orow.ctypes.data_as(ctypes.c_void_p),
                                              ocol.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(n)))
    return orow[:n.value].copy(), ocol[:n.value].copy(), oval[:n.value].copy()


def restrict(m: MasPcg, mapping: GalerkinMapping, fine_rhs):
    """b_c = P^T b (maspcg_galerkin_restrict)."""
    g, keep = mapping._struct()
    f = np.ascontiguousarray(fine_rhs, np.float64)
    out = np.zeros(3 * mapping.coarse_blocks)
    m._ck(m.lib.maspcg_galerkin_restrict(m.h, ctypes.byref(g), f.ctypes.data_as(ctypes.c_void_p),
                                         out.ctypes.data_as(ctypes.c_void_p)))
    return out


def prolong(m: MasPcg, mapping: GalerkinMapping, coarse_x):
    """x = P x_c (maspcg_galerkin_prolong)."""
    g, keep = mapping._struct()
    cx = np.ascontiguousarray(coarse_x, np.float64)
    out = np.zeros(3 * mapping.fine_blocks)
    m._ck(m.lib.maspcg_galerkin_prolong(m.h, ctypes.byref(g), cx.ctypes.data_as(ctypes.c_void_p),
                                        out.ctypes.data_as(ctypes.c_void_p)))
    return out


def coarse_solve(mapping: GalerkinMapping, rows, cols, values9, fine_rhs, *, tolerance=1e-3,
                 max_iterations=None, **cfg):
    """The coarse direction P A_c^-1 P^T b: Galerkin assembly, MAS32 + PCG on
    the coarse system (Euclidean gate at `tolerance`), prolongation.  Returns
    (fine_direction, coarse_x, result dict)."""
    from .frozen_io import CoarseSnapshot, solve_coarse_snapshot
    with MasPcg() as m:
        cr, cc, cv = coarse_matrix(m, mapping, rows, cols, values9)
        bc = restrict(m, mapping, fine_rhs)
        n = mapping.coarse_blocks
        limit = max_iterations if max_iterations is not None else min(512, 3 * n)
        meta = {"format": "agipc_coarse_system_v1", "coarse_block_nodes": n, "coarse_unique_blocks": len(cr),
                "coarse_matrix_half_storage": True,
                "coarse_solve": {"max_iterations": int(limit), "relative_tolerance": float(tolerance)}}
        snap = CoarseSnapshot(meta, cr, cc, cv, bc, np.zeros(3 * n))
        xc, res = solve_coarse_snapshot(snap, **cfg)
        x = prolong(m, mapping, xc)
    return x, xc, res
