"""Shared fixtures for the parity tests (systems and reference restatements)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def spmv_kat_system():
    """The self-test system of run_spmv_equivalence_self_test (spmv.cu:301-346):
    20 block rows, dense lower triangle, hand-formula blocks, a=1.25, b=-0.5."""
    block_rows = 20
    vals, rows, cols = [], [], []
    for i in range(block_rows):
        for j in range(i + 1):
            if i == j:
                B = np.array([[6.0 + i, 0.03, -0.02], [0.03, 7.0 + i, 0.01], [-0.02, 0.01, 8.0 + i]])
            else:
                s = 0.02 * (i + j + 1)
                B = np.array([[s, -0.5 * s, 0.25 * s], [0.4 * s, -0.3 * s, 0.1 * s], [-0.2 * s, 0.35 * s, 0.6 * s]])
            vals.append(B.T.reshape(9))  # Eigen column-major
            rows.append(i)
            cols.append(j)
    dof = 3 * block_rows
    x = np.array([0.125 * (i + 1) - 0.4 for i in range(dof)])
    y0 = np.array([0.05 * (i - 3) for i in range(dof)])
    return np.array(vals), np.array(rows, np.int32), np.array(cols, np.int32), x, y0, 1.25, -0.5


def spmv_kat_expected(vals, rows, cols, x, y0, a, b):
    """The CPU reference loop of the self-test (spmv.cu:348-364)."""
    ref = b * y0.copy()
    for k in range(len(rows)):
        i, j = rows[k], cols[k]
        B = vals[k].reshape(3, 3).T
        ref[3 * i:3 * i + 3] += a * B @ x[3 * j:3 * j + 3]
        if i != j:
            ref[3 * j:3 * j + 3] += a * B.T @ x[3 * i:3 * i + 3]
    return ref


def hierarchy_kat_inputs():
    """run_hierarchy_self_test (TraditionalMAS32Preconditioner.cu:257-296):
    35 valid nodes in 64 padded slots, two chains (0..31) and (32..34)."""
    valid, padded = 35, 64
    start, num, lst = [], [], []
    for v in range(valid):
        start.append(len(lst))
        gb, ge = (0, 32) if v < 32 else (32, valid)
        if v > gb:
            lst.append(v - 1)
        if v + 1 < ge:
            lst.append(v + 1)
        num.append(len(lst) - start[-1])
    pmr = np.full(padded, -1, np.int32)
    pmr[:valid] = np.arange(valid)
    rmp = np.arange(valid, dtype=np.int32)
    return valid, np.array(start, np.uint32), np.array(num, np.uint32), np.array(lst, np.uint32), pmr, rmp


def hierarchy_kat_expected():
    """Expectations of :396-414."""
    valid = 35
    mask = np.array([0xFFFFFFFF if v < 32 else 0x7 for v in range(valid)], np.uint32)
    coarse = np.array([0 if v < 32 else 1 for v in range(valid)], np.int32)
    return {"fine_mask": mask, "coarse": coarse, "going_next": 64 + coarse, "prefix": [1, 1], "level_size1": (2, 64)}


def load_kat257():
    d = os.path.join(GOLDEN, "kat257")
    meta = json.load(open(os.path.join(d, "metadata.json")))
    n, u = meta["coarse_block_nodes"], meta["coarse_unique_blocks"]
    vals = np.fromfile(os.path.join(d, "coarse_A_values.f64x9.bin")).reshape(u, 9)
    rows = np.fromfile(os.path.join(d, "coarse_A_rows.i32.bin"), np.int32)
    cols = np.fromfile(os.path.join(d, "coarse_A_cols.i32.bin"), np.int32)
    rhs = np.fromfile(os.path.join(d, "coarse_rhs.f64.bin"))
    ref = np.fromfile(os.path.join(d, "coarse_solution.f64.bin"))
    published = json.load(open(os.path.join(d, "published.json")))
    cpu = json.load(open(os.path.join(d, "reference_cpu_replay.json")))
    return meta, vals, rows, cols, rhs, ref, published, cpu


def kat257_padded():
    """replay_coarse_snapshot's preparation (agipc_coarse_replay.cu:215-310):
    pad to a multiple of 32 with identity blocks, neighbour graph from the
    matrix pattern (sorted, unique), identity partition maps."""
    meta, vals, rows, cols, rhs, ref, published, cpu = load_kat257()
    n = meta["coarse_block_nodes"]
    padded = (n + 31) // 32 * 32
    eye9 = np.eye(3).T.reshape(9)
    vals_p = np.concatenate([vals, np.tile(eye9, (padded - n, 1))])
    rows_p = np.concatenate([rows, np.arange(n, padded, dtype=np.int32)])
    cols_p = np.concatenate([cols, np.arange(n, padded, dtype=np.int32)])
    graph = [set() for _ in range(padded)]
    for r, c in zip(rows, cols):
        if r != c:
            graph[r].add(int(c))
            graph[c].add(int(r))
    start, num, lst = [], [], []
    for i in range(padded):
        a = sorted(graph[i])
        start.append(len(lst))
        num.append(len(a))
        lst += a
    ident = np.arange(padded, dtype=np.int32)
    return dict(n=n, padded=padded, vals=vals_p, rows=rows_p, cols=cols_p,
                rhs=np.concatenate([rhs, np.zeros(3 * (padded - n))]), ref=np.concatenate([ref, np.zeros(3 * (padded - n))]),
                start=np.array(start, np.uint32), num=np.array(num, np.uint32), lst=np.array(lst, np.uint32),
                ident=ident, published=published, cpu=cpu, limit=min(512, 3 * n))


def permute_full_bcsr(nb_int, iof, rowptr, col, vals):
    """Oracle full BCSR (original rows) renumbered into the internal order."""
    nb = len(rowptr) - 1
    out_rows = [[] for _ in range(nb_int)]
    for r in range(nb):
        ri = iof[r]
        for t in range(rowptr[r], rowptr[r + 1]):
            out_rows[ri].append((iof[col[t]], vals[t]))
    rp = np.zeros(nb_int + 1, np.int64)
    cs, vs = [], []
    for ri in range(nb_int):
        ent = sorted(out_rows[ri], key=lambda e: e[0])
        rp[ri + 1] = rp[ri] + len(ent)
        for c, v in ent:
            cs.append(c)
            vs.append(v.reshape(3, 3).T.reshape(9))  # column-major -> row-major
    return rp, np.array(cs, np.int64), np.array(vs).reshape(-1, 9) if vs else np.zeros((0, 9))


def unpack_domain(packed):
    """96x96 symmetric matrix from a domain's 528 packed upper 3x3 blocks
    (block (a, b), a <= b, at 32a - a(a+1)/2 + b; column-major blocks)."""
    p = np.asarray(packed, np.float64).reshape(528, 9)
    A = np.zeros((96, 96))
    for a in range(32):
        for b in range(a, 32):
            blk = p[32 * a - a * (a + 1) // 2 + b].reshape(3, 3).T
            A[3 * a:3 * a + 3, 3 * b:3 * b + 3] = blk
            A[3 * b:3 * b + 3, 3 * a:3 * a + 3] = blk.T
    return A


def expand_unused(A):
    """A with every zero diagonal entry set to 1 (unused domain slots)."""
    A = A.copy()
    d = np.diag(A).copy()
    d[d == 0] = 1.0
    np.fill_diagonal(A, d)
    return A


def _round_bf16(v):
    f = np.asarray(v, np.float32)
    bits = f.view(np.uint32).astype(np.uint64)
    bits = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    return bits.astype(np.uint32).view(np.float32).astype(np.float64)


def factored_inverse_16(A, kind):
    """A^-1 = W^T W with W = L^-1 (A = L L^T), W stored column-scaled in a
    16-bit type: W = V S, S_j = max_i |W_ij|, V rounded; returns S V^T V S.
    Zero diagonal entries (unused slots) are set to 1 first, as the kernel does."""
    L = np.linalg.cholesky(expand_unused(A))
    W = np.linalg.inv(L)
    S = np.abs(W).max(axis=0)
    S[S == 0] = 1.0
    V = W / S
    V = _round_bf16(V) if kind == "bf16" else V.astype(np.float16).astype(np.float64)
    Wr = V * S
    return Wr.T @ Wr


def inverse_residual(A, M):
    """Root-mean-square entry of A M - I (the oracle's local check)."""
    R = A @ M - np.eye(A.shape[0])
    return float(np.sqrt((R * R).sum() / A.shape[0]))
