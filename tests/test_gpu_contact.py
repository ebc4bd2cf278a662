"""Contact-pair dedup and boundary clearing on the GPU, bit-exact against the
oracle's restatement (GIPC.cu:10130-10181), through the C ABI."""
import numpy as np
import pytest

import oracle
from agipc_learning_b200 import _native as N
from agipc_learning_b200.solver import MasPcg
from tests.test_contact_cpu import _contact_triplets

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,nv,seed", [(1, 4, 1), (31, 20, 2), (33, 20, 3), (200_000, 60_000, 4)])
def test_adjust_contacts_bit_exact_host_arrays(n, nv, seed):
    rows, cols, vals, bd = _contact_triplets(n, nv, seed)
    er, ec, ev, bad = oracle.adjust_contacts(rows, cols, vals, bd, offset=16)
    assert bad == -1
    r, c, v = rows.copy(), cols.copy(), vals.copy()
    with MasPcg(preconditioner="none") as m:
        m.adjust_contact_triplets(r, c, v, bd, 16)
    assert np.array_equal(r, er) and np.array_equal(c, ec)
    assert np.array_equal(v.view(np.uint64), ev.view(np.uint64))


def test_adjust_contacts_bit_exact_device_arrays():
    import torch
    rows, cols, vals, bd = _contact_triplets(100_003, 20_000, 9)
    er, ec, ev, _ = oracle.adjust_contacts(rows, cols, vals, bd, offset=-5)
    r, c = torch.from_numpy(rows.copy()).cuda(), torch.from_numpy(cols.copy()).cuda()
    v, b = torch.from_numpy(vals.copy()).cuda(), torch.from_numpy(bd).cuda()
    with MasPcg(preconditioner="none") as m:
        m.adjust_contact_triplets(r, c, v, b, -5)
    torch.cuda.synchronize()
    assert np.array_equal(r.cpu().numpy(), er) and np.array_equal(c.cpu().numpy(), ec)
    assert np.array_equal(v.cpu().numpy().view(np.uint64), ev.view(np.uint64))


def test_adjust_contacts_rejects_out_of_range_vertex():
    rows, cols, vals, bd = _contact_triplets(1000, 100, 5, bad=3)
    r, c, v = rows.copy(), cols.copy(), vals.copy()
    with MasPcg(preconditioner="none") as m:
        with pytest.raises(N.MaspcgError) as e:
            m.adjust_contact_triplets(r, c, v, bd, 0)
        assert e.value.status == N.ERR_INVALID_ARGUMENT
    er, ec, ev, _ = oracle.adjust_contacts(rows, cols, vals, bd, offset=0)
    assert np.array_equal(r, er) and np.array_equal(c, ec) and np.array_equal(v, ev)


def test_zero_boundary_bit_exact():
    rows, cols, vals, bd = _contact_triplets(150_000, 30_000, 6)
    off = 40
    ev, _ = oracle.zero_boundary(rows + off, cols + off, vals, bd, off)
    v = vals.copy()
    with MasPcg(preconditioner="none") as m:
        m.zero_boundary_triplets(rows + off, cols + off, v, bd, off)
    assert np.array_equal(v.view(np.uint64), ev.view(np.uint64))


def test_adjusted_contacts_merge_like_the_reference():
    """A barrier's full 4x4 pattern (both (a, b) and (b, a)) through the
    adjust step and the merge gives each coupling once: the merged system
    equals the one built from the upper blocks alone."""
    rng = np.random.default_rng(21)
    nv, pairs = 400, 300
    rows, cols, vals = [], [], []
    upper = {}
    for _ in range(pairs):
        vs = rng.choice(nv, 4, replace=False)
        H = rng.standard_normal((12, 12))
        H = H @ H.T
        for i in range(4):
            for j in range(4):
                blk = H[3 * i:3 * i + 3, 3 * j:3 * j + 3]
                rows.append(vs[i])
                cols.append(vs[j])
                vals.append(blk.T.reshape(9))  # column-major
                if vs[i] <= vs[j]:
                    key = (int(vs[i]), int(vs[j]))
                    upper[key] = upper.get(key, 0) + blk
    rows, cols, vals = np.array(rows, np.int32), np.array(cols, np.int32), np.array(vals)
    bd = np.zeros(nv, np.int32)
    with MasPcg(preconditioner="none") as m:
        m.adjust_contact_triplets(rows, cols, vals, bd, 0)
        ur, uc, uv = m.convert_bcoo(rows, cols, vals)
    got = {(int(a), int(b)): v.reshape(3, 3).T for a, b, v in zip(ur, uc, uv)}
    assert set(got) == set(upper)
    for k, blk in upper.items():
        assert np.allclose(got[k], blk, rtol=0, atol=1e-12 * np.abs(blk).max())
