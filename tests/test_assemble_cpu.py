"""The CPU restatements of the triplet merge (Converter::convert,
linear_system/utils/converter.cu:137-284) and of the contact-triplet
partition (GIPC::partitionContactHessian, GIPC.cu:9952-10128) against
plain numpy formulations of the same contracts."""
import numpy as np
import pytest

import oracle


def _triplets(rng, n, nb, dup):
    rows = rng.integers(0, nb, n).astype(np.int32)
    cols = rng.integers(0, nb, n).astype(np.int32)
    lo, hi = np.minimum(rows, cols), np.maximum(rows, cols)
    if dup and n > 4:  # repeat a third of the keys
        k = n // 3
        lo[-k:], hi[-k:] = lo[:k], hi[:k]
    return lo, hi, rng.standard_normal((n, 9))


@pytest.mark.parametrize("n,nb,dup", [(0, 5, False), (1, 5, False), (500, 40, True), (5000, 10, True)])
def test_convert_oracle_matches_numpy(n, nb, dup):
    rng = np.random.default_rng(n + nb)
    r, c, v = _triplets(rng, n, nb, dup)
    orow, ocol, oval = oracle.convert_triplets(r, c, v)
    key = (r.astype(np.uint64) << np.uint64(32)) + c.astype(np.uint64)
    order = np.argsort(key, kind="stable")
    uk, first = np.unique(key[order], return_index=True)
    assert np.array_equal(orow, (uk >> np.uint64(32)).astype(np.int32))
    assert np.array_equal(ocol, (uk & np.uint64(0xffffffff)).astype(np.int32))
    ref = np.zeros((len(uk), 9))
    bounds = list(first) + [n]
    for u in range(len(uk)):
        acc = np.zeros(9)
        for t in order[bounds[u]:bounds[u + 1]]:  # sequential, stable order
            acc = acc + v[t]
        ref[u] = acc
    assert np.array_equal(oval, ref)


@pytest.mark.parametrize("n", [0, 1, 7, 2000])
def test_partition_oracle_matches_numpy(n):
    rng = np.random.default_rng(n)
    r, c, v = _triplets(rng, n, 50, False)
    t = rng.integers(0, 4, n).astype(np.uint64)
    orow, ocol, oval, counts = oracle.partition_contacts(r, c, v, t)
    order = np.argsort(t, kind="stable")
    assert np.array_equal(orow, r[order]) and np.array_equal(ocol, c[order]) and np.array_equal(oval, v[order])
    assert np.array_equal(counts, np.bincount(t.astype(np.int64), minlength=4))


def test_partition_oracle_rejects_unknown_type():
    with pytest.raises(ValueError):
        oracle.partition_contacts([0], [0], np.zeros((1, 9)), np.array([4], np.uint64))
