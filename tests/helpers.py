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


def unpack_domain(packed, bank=32):
    """3B x 3B symmetric matrix from a domain's B(B+1)/2 packed upper 3x3
    blocks (block (a, b), a <= b, at Ba - a(a+1)/2 + b; column-major blocks)."""
    B = bank
    p = np.asarray(packed, np.float64).reshape(B * (B + 1) // 2, 9)
    A = np.zeros((3 * B, 3 * B))
    for a in range(B):
        for b in range(a, B):
            blk = p[B * a - a * (a + 1) // 2 + b].reshape(3, 3).T
            A[3 * a:3 * a + 3, 3 * b:3 * b + 3] = blk
            A[3 * b:3 * b + 3, 3 * a:3 * a + 3] = blk.T
    return A


def _decode_pairs(pairs, node_offset, nv):
    """FEM-local vertex tuples of int4 contact pairs (the sign encoding of
    _buildCollisionConnection_new)."""
    out = []
    for x, y, z, w in np.asarray(pairs, np.int64).reshape(-1, 4):
        if x >= 0:
            v = [x, y, z, -w - 1 if w < 0 else w]
        else:
            x = -x - 1
            if z < 0:
                v = [x, -y - 1, -z - 1, -w - 1] if y < 0 else [x, y]
            elif w < 0:
                v = [x, -y - 1, z, -w - 1] if y < 0 else [x, y, z]
            else:
                v = [x, y, z, w]
        loc = [int(t) - node_offset for t in v]
        out.append([t for t in loc if 0 <= t < nv])
    return out


def mas_levels(s, bank):
    """The MAS hierarchy by its meaning, independent of the mask kernels: the
    nodes of level l+1 are the connected components, inside each bank of B
    consecutive level-l nodes, of the graph of mesh edges and contact pairs;
    they are numbered bank by bank, inside a bank by their lowest lane.
    Level 0 nodes are the partition slots.  Returns fine_mask, per-level
    node ids (levels 1..L), level sizes [L+1, 2] and components per level-0
    bank."""
    import oracle
    B = bank
    nv, pmr, rmp = s.fem_count, np.asarray(s.part_map_real), np.asarray(s.real_map_part)
    L = oracle.compute_num_levels(max(len(pmr), nv), bank)
    st, nn, nl = (np.asarray(a) for a in (s.neighbor_start, s.neighbor_num, s.neighbor_list))
    edges = [(v, int(u)) for v in range(nv) for u in nl[st[v]:st[v] + nn[v]]]
    for grp in _decode_pairs(s.pairs, s.node_offset, nv):
        edges += [(grp[i], grp[j]) for i in range(len(grp)) for j in range(i + 1, len(grp))]
    node = rmp.astype(np.int64).copy()  # level-0 node = slot
    count, begin = len(pmr), 0
    ids, sizes = [], [(len(pmr), 0)]
    fine_mask = prefix = None
    for level in range(L):
        parent = list(range(count))

        def find(a):
            while parent[a] != a:
                parent[a] = parent[parent[a]]
                a = parent[a]
            return a
        for u, v in edges:
            a, b = int(node[u]), int(node[v])
            if a // B == b // B and a != b:
                ra, rb = find(a), find(b)
                if ra != rb:
                    parent[max(ra, rb)] = min(ra, rb)  # root: lowest member
        live = np.zeros(count, bool)
        live[node] = True
        new = np.full(count, -1, np.int64)
        comps = np.zeros((count + B - 1) // B, np.int64)
        nxt = 0
        for a in range(count):
            if live[a] and find(a) == a:
                new[a] = nxt
                comps[a // B] += 1
                nxt += 1
        for a in range(count):
            if live[a]:
                new[a] = new[find(a)]
        if level == 0:
            fine_mask = np.zeros(nv, np.uint32)
            for v in range(nv):
                a = node[v]
                for u in range(a - a % B, a - a % B + B):
                    if u < count and live[u] and find(u) == find(a):
                        fine_mask[v] |= np.uint32(1 << (u % B))
            prefix = comps
        begin += (count + B - 1) // B * B
        node = new[node]
        ids.append(node.copy())
        count = nxt
        sizes.append((count, begin))
    return {"fine_mask": fine_mask, "ids": np.array(ids), "level_size": np.array(sizes), "prefix": prefix,
            "levelnum": L}


def galerkin_domains(s, lev, bank, cemas16):
    """Packed upper FP64 domain matrices of every level by their meaning: the
    Galerkin sum over the FEM entries A_ij whose level-l nodes share a bank,
    minus the entries CEMAS16 leaves out (cemas16=True): an in-bank pair of
    level-0 slots whose order runs against the vertex order, and, above
    level 0, the in-bank entries of a row whose even partner slot is padding
    when the bank is one component."""
    B = bank
    nv, fo = s.fem_count, s.fem_offset
    pmr, rmp = np.asarray(s.part_map_real), np.asarray(s.real_map_part)
    L = lev["levelnum"]
    begins = [0] + [int(lev["level_size"][l][1]) for l in range(1, L)]
    total = int(lev["level_size"][L][1])
    P = B * (B + 1) // 2
    out = np.zeros((total // B, P, 9))
    r, c, v = np.asarray(s.rows), np.asarray(s.cols), np.asarray(s.vals).reshape(-1, 3, 3).transpose(0, 2, 1)
    sel = (r >= fo) & (r < fo + nv) & (c >= fo) & (c < fo + nv)
    ent = []
    for i, j, blk in zip(r[sel] - fo, c[sel] - fo, v[sel]):
        ent.append((i, j, blk))
        if i != j:
            ent.append((j, i, blk.T))
    for i, j, blk in ent:
        si, sj = rmp[i], rmp[j]
        same0 = si // B == sj // B
        if cemas16 and same0 and i != j and ((i < j) != (si < sj)):
            continue
        for l in range(L):
            if l == 0:
                a, b = si, sj
            else:
                if cemas16 and same0 and lev["prefix"][si // B] == 1 and pmr[si & ~1] < 0:
                    continue
                a, b = begins[l] + lev["ids"][l - 1][i], begins[l] + lev["ids"][l - 1][j]
            if a // B != b // B or a > b:
                continue
            g, la, lb = a // B, a % B, b % B
            out[g, B * la - la * (la + 1) // 2 + lb] += blk.T.reshape(9)  # column-major
    return out


def gapped_partition(s, bank=16, gap=2):
    """Partition of a vertex-sorted system (partition_for_bank) with slot
    `gap` of every bank left empty: B - 1 consecutive vertices per bank."""
    import dataclasses
    nv, B = s.fem_count, bank
    per = B - 1
    nbanks = (nv + per - 1) // per
    pmr = np.full(nbanks * B, -1, np.int32)
    rmp = np.zeros(nv, np.int32)
    for v in range(nv):
        b, k = divmod(v, per)
        slot = b * B + (k if k < gap else k + 1)
        pmr[slot] = v
        rmp[v] = slot
    return dataclasses.replace(s, part_map_real=pmr, real_map_part=rmp, name=s.name + "_gap")


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


def compare_hierarchy(g, o):
    """GPU hierarchy (MasPcg.hierarchy) equals the oracle's, bit for bit."""
    L = o["levelnum"]
    assert g["levelnum"] == L
    assert np.array_equal(g["fine_mask"], o["fine_mask"])
    assert np.array_equal(g["coarse_space_tables"], o["coarse_space_tables"])
    assert np.array_equal(g["going_next"], o["going_next"])
    assert np.array_equal(g["level_size"][1:], o["level_size"][1:])
    assert np.array_equal(g["coarse_table"][:, :L - 1], o["coarse_table"][:, :L - 1])
    assert np.array_equal(g["prefix_original"], o["prefix_original"])
    assert g["total_clusters"] == o["total_clusters"]


def load_cfg0_replay():
    """The reference's CPU block-Jacobi replay of config 0 (tests/golden/cfg0_replay,
    made by tests/golden/make_golden.py): (its report for the sample, the
    SHA-256 of the exported snapshot arrays)."""
    d = os.path.join(GOLDEN, "cfg0_replay")
    report = json.load(open(os.path.join(d, "reference_cpu_replay.json")))["samples"][0]
    return report, json.load(open(os.path.join(d, "manifest.json")))["sha256"]


def cfg0_snapshot_sums():
    """Config 0 regenerated and written as the golden generator writes it;
    the SHA-256 of each array file."""
    import importlib.util
    import tempfile

    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    with tempfile.TemporaryDirectory() as tmp:
        return mg.cfg0_snapshot(os.path.join(tmp, "cfg0"))


def direct_solution(s):
    """x = A^-1 b by SciPy's sparse LU (the replay's --direct-reference)."""
    from scipy.sparse.linalg import spsolve

    from oracle.mixed_emulation import full_matrix

    return spsolve(full_matrix(s).tocsc(), s.b)
