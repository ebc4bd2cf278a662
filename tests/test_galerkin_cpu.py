"""The Galerkin coarse-space restatement (oracle.galerkin_expand;
StiffGIPC/agipc/agipc_galerkin.cu:200-283) pinned on the reference's own
known-answer test, galerkin_self_test (agipc_galerkin.cu:1417-1470): a
formula-defined SPD fine matrix on 7 blocks (one prefix block, six FEM nodes:
four in an affine coarse node, two in a translational one), whose coarse
matrix must equal P^T A P of the dense prolongation."""
import numpy as np

import oracle


def kat():
    """The inputs of galerkin_self_test, rebuilt from its formulas."""
    fb, prefix = 7, 1
    q = np.array([[np.sin(0.31 * (r + 1) * (c + 2)) + 0.2 * np.cos(0.17 * (r + 3 + c)) for c in range(3 * fb)]
                  for r in range(3 * fb)])
    dense = q.T @ q + np.eye(3 * fb)
    rows, cols, vals = [], [], []
    for r in range(fb):
        for c in range(r, fb):
            rows.append(r)
            cols.append(c)
            vals.append(dense[3 * r:3 * r + 3, 3 * c:3 * c + 3].T.reshape(9))  # Eigen column-major
    mapping = dict(prefix=prefix, fine_to_coarse=np.array([0, 0, 0, 0, 1, 1], np.int32),
                   bases=np.array([1, 0], np.int32), masks=np.array([15, 1], np.int32),
                   rest=np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [-0.1, 0.8, -0.6], [0.9, 0.4, 0.2]],
                                 np.float64), coarse_block_nodes=5)
    b = 0.25 + 0.125 * np.arange(3 * fb)
    return dense, (np.array(rows, np.int32), np.array(cols, np.int32), np.array(vals)), mapping, b


def dense_from_upper(rows, cols, vals, n):
    A = np.zeros((3 * n, 3 * n))
    for r, c, v in zip(rows, cols, vals):
        B = np.asarray(v).reshape(3, 3).T
        A[3 * r:3 * r + 3, 3 * c:3 * c + 3] += B
        if r != c:
            A[3 * c:3 * c + 3, 3 * r:3 * r + 3] += B.T
    return A


def test_galerkin_kat_coarse_matrix_is_pt_a_p():
    dense, (r, c, v), mp, b = kat()
    er, ec, ev = oracle.galerkin_expand(r, c, v, mp["prefix"], mp["fine_to_coarse"], mp["bases"], mp["masks"],
                                        mp["rest"])
    cr, cc, cv = oracle.convert_triplets(er, ec, ev)
    assert np.all(cr <= cc)
    nc = mp["prefix"] + mp["coarse_block_nodes"]
    P = oracle.galerkin_prolongation(7, nc, mp["prefix"], mp["fine_to_coarse"], mp["bases"], mp["masks"],
                                     mp["rest"])
    expected = P.T @ dense @ P
    actual = dense_from_upper(cr, cc, cv, nc)
    # the reference's gate: ||actual - expected||_F / max(1, ||expected||_F)
    assert np.linalg.norm(actual - expected) / max(1.0, np.linalg.norm(expected)) <= 1e-12
    # coarse direction of the KAT
    xc = np.linalg.solve(expected, P.T @ b)
    assert np.linalg.norm(P @ xc) > 0
