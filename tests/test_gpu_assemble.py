"""The triplet merge and the contact-triplet partition on the GPU, through
the C ABI, against the CPU restatements: bit-exact (integer structure and
the FP64 sums, which both add a key's blocks in input order)."""
import numpy as np
import pytest

import oracle
from agipc_learning_b200 import synth
from agipc_learning_b200.solver import MasPcg

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def handle():
    with MasPcg() as m:
        yield m


def _triplets(rng, n, nb, dup):
    rows = rng.integers(0, nb, n).astype(np.int32)
    cols = rng.integers(0, nb, n).astype(np.int32)
    lo, hi = np.minimum(rows, cols), np.maximum(rows, cols)
    if dup and n > 4:
        k = n // 3
        lo[-k:], hi[-k:] = lo[:k], hi[:k]
    return lo, hi, rng.standard_normal((n, 9))


@pytest.mark.parametrize("n,nb,dup", [(1, 3, False), (700, 30, True), (200_000, 5_000, True)])
def test_convert_bcoo_bit_exact(handle, n, nb, dup):
    rng = np.random.default_rng(n)
    r, c, v = _triplets(rng, n, nb, dup)
    orow, ocol, oval = oracle.convert_triplets(r, c, v)
    grow, gcol, gval = handle.convert_bcoo(r, c, v)          # host arrays
    assert np.array_equal(grow, orow) and np.array_equal(gcol, ocol) and np.array_equal(gval, oval)
    dev = torch.device("cuda")
    trow, tcol, tval = handle.convert_bcoo(torch.tensor(r, device=dev), torch.tensor(c, device=dev),
                                           torch.tensor(v, device=dev))  # device arrays
    assert np.array_equal(trow.cpu().numpy(), orow) and np.array_equal(tval.cpu().numpy(), oval)


def test_convert_bcoo_of_a_raw_assembly(handle):
    """The 32^3 per-tet-modulus system's raw triplets (10 per tet, mass, in
    element order) merge to the generator's own matrix."""
    s = synth.config_system(3)
    R, C, V = s.meta["raw"]
    grow, gcol, gval = handle.convert_bcoo(R, C, V)
    orow, ocol, oval = oracle.convert_triplets(R, C, V)
    assert np.array_equal(grow, orow) and np.array_equal(gcol, ocol) and np.array_equal(gval, oval)
    key = lambda a, b: (np.asarray(a, np.int64) << 32) + np.asarray(b, np.int64)  # noqa: E731
    o = np.argsort(key(s.rows, s.cols))
    assert np.array_equal(key(grow, gcol), key(s.rows, s.cols)[o])
    assert np.abs(gval - s.vals[o]).max() <= 1e-12 * np.abs(s.vals).max()


def test_convert_bcoo_rejects_negative_index_and_stays_usable(handle):
    v = np.zeros((2, 9))
    with pytest.raises(RuntimeError):
        handle.convert_bcoo(np.array([0, -1], np.int32), np.array([0, 0], np.int32), v)
    r, c, vv = handle.convert_bcoo(np.array([1, 1], np.int32), np.array([2, 2], np.int32), np.ones((2, 9)))
    assert list(r) == [1] and list(c) == [2] and np.all(vv == 2.0)


def test_convert_bcoo_empty(handle):
    r, c, v = handle.convert_bcoo(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros((0, 9)))
    assert len(r) == 0


@pytest.mark.parametrize("n,types", [(1, (2,)), (5000, (0, 1, 2, 3)), (3000, (0, 3)), (100_000, (1,))])
def test_partition_contact_triplets_bit_exact(handle, n, types):
    rng = np.random.default_rng(n + len(types))
    r, c, v = _triplets(rng, n, 1000, False)
    t = rng.choice(np.array(types, np.uint64), n)
    orow, ocol, oval, ocount = oracle.partition_contacts(r, c, v, t)
    grow, gcol, gval, gcount = handle.partition_contact_triplets(r, c, v, t)
    assert np.array_equal(gcount, ocount)
    assert np.array_equal(grow, orow) and np.array_equal(gcol, ocol) and np.array_equal(gval, oval)


def test_partition_rejects_unknown_type(handle):
    with pytest.raises(RuntimeError):
        handle.partition_contact_triplets(np.zeros(2, np.int32), np.zeros(2, np.int32), np.zeros((2, 9)),
                                          np.array([0, 7], np.uint64))
