"""Frozen Newton systems and coarse snapshots in the reference's file formats.

Two on-disk formats written by StiffGIPC, both raw little-endian arrays:

* A frozen Newton system (GlobalLinearSystem's dump,
  StiffGIPC/linear_system/linear_system/global_linear_system.cu:380-402):
  ``frozen_A_values.bin`` (9 doubles per block, Eigen column-major),
  ``frozen_A_rows.bin`` / ``frozen_A_cols.bin`` (int32 block indices) and
  ``frozen_b.bin`` (doubles, 3 per block row).  The block list is the triplet
  matrix as assembled, upper blocks (row <= col), repeats allowed.
* A coarse snapshot (``agipc_coarse_system_v1``;
  StiffGIPC/agipc/agipc_coarse_replay.cu:196-213 and
  reports/agipc_reproduction/replay_frozen_coarse.py:24-67): ``metadata.json``
  with ``coarse_block_nodes``, ``coarse_unique_blocks``,
  ``coarse_matrix_half_storage`` and ``coarse_solve`` {max_iterations,
  relative_tolerance}; ``coarse_A_values.f64x9.bin``, ``coarse_A_rows.i32.bin``,
  ``coarse_A_cols.i32.bin``, ``coarse_rhs.f64.bin`` and
  ``coarse_solution.f64.bin``.

`coarse_replay_inputs` prepares a snapshot the way replay_coarse_snapshot
does (agipc_coarse_replay.cu:215-310): pad the block count to a multiple of
32 with identity blocks, build the neighbour graph from the matrix pattern
(sorted, unique, symmetric) and use the identity partition, so that MAS32
treats every 32 consecutive blocks as one domain.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass

import numpy as np

FROZEN_FILES = ("frozen_A_values.bin", "frozen_A_rows.bin", "frozen_A_cols.bin", "frozen_b.bin")


@dataclass
class FrozenSystem:
    rows: np.ndarray   # int32 [n]
    cols: np.ndarray   # int32 [n]
    vals: np.ndarray   # float64 [n, 9], Eigen column-major
    b: np.ndarray      # float64 [3 * block_rows]

    @property
    def block_rows(self) -> int:
        return len(self.b) // 3


def _read(path: str, dtype, count: int | None = None) -> np.ndarray:
    a = np.fromfile(path, dtype=dtype)
    if count is not None and a.size != count:
        raise ValueError(f"{path}: {a.size} values, expected {count}")
    if np.issubdtype(a.dtype, np.floating) and not np.all(np.isfinite(a)):
        raise ValueError(f"{path}: nonfinite data")
    return a


def read_frozen(directory: str) -> FrozenSystem:
    """A frozen Newton system written by the reference's dump."""
    v, r, c, b = (os.path.join(directory, f) for f in FROZEN_FILES)
    rows = _read(r, np.int32)
    cols = _read(c, np.int32, rows.size)
    vals = _read(v, np.float64, 9 * rows.size).reshape(-1, 9)
    rhs = _read(b, np.float64)
    if rhs.size % 3:
        raise ValueError(f"{b}: length {rhs.size} is not a multiple of 3")
    nb = rhs.size // 3
    if rows.size and (rows.min() < 0 or cols.min() < 0 or rows.max() >= nb or cols.max() >= nb):
        raise ValueError("frozen matrix index out of bounds")
    return FrozenSystem(rows, cols, vals, rhs)


def write_frozen(directory: str, rows, cols, vals, b) -> None:
    os.makedirs(directory, exist_ok=True)
    arrays = (np.ascontiguousarray(vals, np.float64).reshape(-1, 9), np.ascontiguousarray(rows, np.int32),
              np.ascontiguousarray(cols, np.int32), np.ascontiguousarray(b, np.float64))
    for name, a in zip(FROZEN_FILES, arrays):
        a.tofile(os.path.join(directory, name))


@dataclass
class CoarseSnapshot:
    metadata: dict
    rows: np.ndarray
    cols: np.ndarray
    vals: np.ndarray
    rhs: np.ndarray
    solution: np.ndarray

    @property
    def blocks(self) -> int:
        return int(self.metadata["coarse_block_nodes"])


def read_coarse_snapshot(directory: str) -> CoarseSnapshot:
    meta = json.load(open(os.path.join(directory, "metadata.json")))
    blocks, unique = int(meta["coarse_block_nodes"]), int(meta["coarse_unique_blocks"])
    if blocks <= 0 or unique <= 0:
        raise ValueError("empty coarse matrix")
    if not meta.get("coarse_matrix_half_storage", True):
        raise ValueError("only symmetric half-storage coarse snapshots are supported")
    p = lambda f: os.path.join(directory, f)  # noqa: E731
    vals = _read(p("coarse_A_values.f64x9.bin"), np.float64, 9 * unique).reshape(unique, 9)
    rows = _read(p("coarse_A_rows.i32.bin"), np.int32, unique)
    cols = _read(p("coarse_A_cols.i32.bin"), np.int32, unique)
    if rows.min() < 0 or cols.min() < 0 or rows.max() >= blocks or cols.max() >= blocks:
        raise ValueError("coarse matrix index out of bounds")
    rhs = _read(p("coarse_rhs.f64.bin"), np.float64, 3 * blocks)
    sol = _read(p("coarse_solution.f64.bin"), np.float64, 3 * blocks)
    return CoarseSnapshot(meta, rows, cols, vals, rhs, sol)


def write_coarse_snapshot(directory: str, snap: CoarseSnapshot) -> None:
    os.makedirs(directory, exist_ok=True)
    meta = dict(snap.metadata)
    meta["coarse_unique_blocks"] = int(len(snap.rows))
    with open(os.path.join(directory, "metadata.json"), "w") as f:
        json.dump(meta, f, indent=2)
    p = lambda f: os.path.join(directory, f)  # noqa: E731
    np.ascontiguousarray(snap.vals, np.float64).tofile(p("coarse_A_values.f64x9.bin"))
    np.ascontiguousarray(snap.rows, np.int32).tofile(p("coarse_A_rows.i32.bin"))
    np.ascontiguousarray(snap.cols, np.int32).tofile(p("coarse_A_cols.i32.bin"))
    np.ascontiguousarray(snap.rhs, np.float64).tofile(p("coarse_rhs.f64.bin"))
    np.ascontiguousarray(snap.solution, np.float64).tofile(p("coarse_solution.f64.bin"))


def coarse_replay_inputs(snap: CoarseSnapshot) -> dict:
    """MasPcg inputs for a coarse snapshot, prepared as replay_coarse_snapshot
    does: identity padding to a multiple of 32 blocks, symmetric sorted
    neighbour graph from the pattern, identity partition."""
    n = snap.blocks
    padded = (n + 31) // 32 * 32
    eye9 = np.eye(3).T.reshape(9)
    vals = np.concatenate([snap.vals, np.tile(eye9, (padded - n, 1))])
    rows = np.concatenate([snap.rows, np.arange(n, padded, dtype=np.int32)])
    cols = np.concatenate([snap.cols, np.arange(n, padded, dtype=np.int32)])
    off = snap.rows != snap.cols
    a = np.concatenate([snap.rows[off], snap.cols[off]]).astype(np.int64)
    b = np.concatenate([snap.cols[off], snap.rows[off]]).astype(np.int64)
    pair = np.unique(a * padded + b)
    src, dst = (pair // padded).astype(np.int64), (pair % padded).astype(np.uint32)
    num = np.bincount(src, minlength=padded).astype(np.uint32)
    start = np.concatenate([[0], np.cumsum(num)[:-1]]).astype(np.uint32)
    ident = np.arange(padded, dtype=np.int32)
    limit = int(snap.metadata.get("coarse_solve", {}).get("max_iterations", min(512, 3 * n)))
    tol = float(snap.metadata.get("coarse_solve", {}).get("relative_tolerance", 1e-3))
    pad = np.zeros(3 * (padded - n))
    return dict(n=n, padded=padded, vals=vals, rows=rows, cols=cols, rhs=np.concatenate([snap.rhs, pad]),
                ref=np.concatenate([snap.solution, pad]), start=start, num=num, lst=dst, ident=ident,
                limit=min(limit, 3 * n), tolerance=tol)


def solve_coarse_snapshot(snap: CoarseSnapshot, **cfg):
    """Replay a coarse snapshot through libmaspcg (MAS32 + PCG, Euclidean gate
    at the snapshot's tolerance).  Returns (x[:3n], result dict)."""
    from .solver import MasPcg
    k = coarse_replay_inputs(snap)
    opts = dict(gate="euclid", tolerance=k["tolerance"], max_iterations=k["limit"] + 1)
    opts.update(cfg)
    with MasPcg(**opts) as m:
        m.set_graph(k["padded"], 0, k["start"], k["num"], k["lst"], k["ident"], k["ident"])
        m.set_contacts(None)
        m.set_matrix(k["vals"], k["rows"], k["cols"], k["padded"])
        m.build()
        x, res = m.solve(k["rhs"])
    return x[:3 * k["n"]], res
