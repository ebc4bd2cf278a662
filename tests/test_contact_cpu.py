"""Contact-pair dedup and boundary clearing (GIPC.cu:10130-10181) and the
Morton partition (gl_main.cu:1178-1242): the oracle's and the generator's C
restatements against independent numpy restatements and hand-computed
cases.  CPU only."""
import numpy as np
import pytest

import oracle
from agipc_learning_b200 import synth


def _contact_triplets(n, nv, seed, bad=0):
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, nv, n).astype(np.int32)
    cols = rng.integers(0, nv, n).astype(np.int32)
    cols[: n // 8] = rows[: n // 8]  # some diagonal blocks
    vals = rng.standard_normal((n, 9))
    bd = (rng.random(nv) < 0.2).astype(np.int32) * rng.integers(1, 4, nv).astype(np.int32)
    if bad:
        pos = rng.choice(n, bad, replace=False)
        rows[pos] = nv + 3
    return rows, cols, vals, bd


def adjust_by_meaning(rows, cols, vals, bd, offset):
    """A lower copy (r > c) moves to the upper slot and is cleared; an upper
    block touching a boundary vertex is cleared; both indices + offset."""
    r, c = rows.astype(np.int64), cols.astype(np.int64)
    lower = r > c
    out_r = np.where(lower, c, r) + offset
    out_c = np.where(lower, r, c) + offset
    clear = lower | (bd[r] != 0) | (bd[c] != 0)
    v = vals.copy()
    v[clear] = 0.0
    return out_r.astype(np.int32), out_c.astype(np.int32), v


def test_adjust_contacts_matches_meaning():
    rows, cols, vals, bd = _contact_triplets(5000, 700, 11)
    r, c, v, bad = oracle.adjust_contacts(rows, cols, vals, bd, offset=8)
    er, ec, ev = adjust_by_meaning(rows, cols, vals, bd, 8)
    assert bad == -1
    assert np.array_equal(r, er) and np.array_equal(c, ec)
    assert np.array_equal(v.view(np.uint64), ev.view(np.uint64))  # bit-exact, +0.0 where cleared
    assert np.all(r <= c)


def test_adjust_contacts_hand_case():
    # vertices 0..3; vertex 2 on the boundary; offset 10 (e.g. 4 ABD bodies - 6 ABD points)
    rows = np.array([0, 1, 3, 2, 1], np.int32)
    cols = np.array([1, 0, 3, 0, 1], np.int32)
    vals = np.arange(45, dtype=np.float64).reshape(5, 9) + 1.0
    bd = np.array([0, 0, 1, 0], np.int32)
    r, c, v, bad = oracle.adjust_contacts(rows, cols, vals, bd, offset=10)
    assert bad == -1
    assert list(r) == [10, 10, 13, 10, 11] and list(c) == [11, 11, 13, 12, 11]
    assert np.array_equal(v[0], vals[0])      # upper, interior: kept
    assert not v[1].any()                      # lower copy of (0, 1): cleared
    assert np.array_equal(v[2], vals[2])      # diagonal, interior: kept
    assert not v[3].any()                      # lower, and touches the boundary vertex
    assert np.array_equal(v[4], vals[4])


def test_adjust_contacts_out_of_range_left_unchanged():
    rows, cols, vals, bd = _contact_triplets(300, 50, 3, bad=4)
    r, c, v, bad = oracle.adjust_contacts(rows, cols, vals, bd, offset=0)
    first = int(np.nonzero(rows >= 50)[0][0])
    assert bad == first
    untouched = rows >= 50
    assert np.array_equal(r[untouched], rows[untouched]) and np.array_equal(v[untouched], vals[untouched])


def test_zero_boundary_matches_meaning():
    rows, cols, vals, bd = _contact_triplets(4000, 500, 5)
    offset = 12
    v, bad = oracle.zero_boundary(rows + offset, cols + offset, vals, bd, offset)
    clear = (bd[rows] != 0) | (bd[cols] != 0)
    ev = vals.copy()
    ev[clear] = 0.0
    assert bad == -1
    assert np.array_equal(v.view(np.uint64), ev.view(np.uint64))


# ----------------------------------------------------------------- Morton --


def _interleave(x, y, z):
    """30-bit code with bit 3k = x bit k, 3k+1 = y bit k, 3k+2 = z bit k."""
    code = 0
    for k in range(10):
        code |= ((x >> k) & 1) << (3 * k) | ((y >> k) & 1) << (3 * k + 1) | ((z >> k) & 1) << (3 * k + 2)
    return code


def morton_by_meaning(X):
    X = np.asarray(X, np.float64)
    lo, hi = X.min(axis=0), X.max(axis=0)
    ext = hi - lo
    with np.errstate(invalid="ignore", divide="ignore"):
        t = np.where(ext > 0, (X - lo) / np.where(ext > 0, ext, 1.0), 0.0)
    q = (np.clip(t, 0.0, 1.0) * 1023.0 + 0.5).astype(np.int64)
    codes = [_interleave(int(a), int(b), int(c)) for a, b, c in q]
    order = sorted(range(len(X)), key=lambda v: (codes[v], v))  # stable: ties by index
    slots = (len(X) + 31) // 32 * 32
    pmr = np.full(slots, -1, np.int32)
    rmp = np.zeros(len(X), np.int32)
    for s, v in enumerate(order):
        pmr[s] = v
        rmp[v] = s
    return pmr, rmp


def test_morton_cube_corners_hand_computed():
    # the 8 corners of the unit cube in a scrambled input order; with one bit
    # per axis the code is x | y << 1 | z << 2 of the top bit pattern, so the
    # order is (0,0,0), (1,0,0), (0,1,0), (1,1,0), (0,0,1), (1,0,1), (0,1,1), (1,1,1)
    corners = [(1, 1, 1), (0, 0, 1), (1, 0, 0), (0, 1, 1), (0, 0, 0), (1, 1, 0), (0, 1, 0), (1, 0, 1)]
    pmr, rmp = synth.morton_partition(np.array(corners, np.float64))
    expect = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0), (0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 1)]
    assert [corners[v] for v in pmr[:8]] == expect
    assert list(pmr[8:]) == [-1] * 24
    assert all(pmr[rmp[v]] == v for v in range(8))


def test_morton_ties_flat_axis_and_rounding():
    X = np.array([
        [0.0, 0.0, 5.0],    # z is flat: every point quantises z to 0
        [1.0, 0.0, 5.0],
        [0.0, 0.0, 5.0],    # tie with point 0: index order
        [0.5, 0.0, 5.0],    # t = 0.5 -> 511.5 + 0.5 = 512 (0b1000000000)
        [0.4995, 0.0, 5.0],  # t * 1023 = 510.99 -> 511 (0b0111111111)
        [0.0, 1.0, 5.0],
    ])
    pmr, rmp = synth.morton_partition(X)
    # codes: p0 = p2 = 0; p4: x = 511 -> interleave of 0x1ff; p3: x = 512 -> bit 27;
    # p1: x = 1023; p5: y = 1023 (bits 1, 4, ...)
    c4, c3, c1, c5 = _interleave(511, 0, 0), _interleave(512, 0, 0), _interleave(1023, 0, 0), _interleave(0, 1023, 0)
    assert c4 < c3 < c1 < c5
    assert list(pmr[:6]) == [0, 2, 4, 3, 1, 5]


@pytest.mark.parametrize("n,seed", [(33, 1), (1000, 2), (4097, 3)])
def test_morton_partition_matches_meaning(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.random((n, 3)) * np.array([2.0, 0.5, 1e-3])
    X[rng.choice(n, n // 10)] = X[0]  # repeated positions: ties
    pmr, rmp = synth.morton_partition(X)
    epmr, ermp = morton_by_meaning(X)
    assert np.array_equal(pmr, epmr) and np.array_equal(rmp, ermp)
