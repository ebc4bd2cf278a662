"""Frozen-system and coarse-snapshot files in the reference's formats (CPU)."""
import os

import numpy as np

from agipc_learning_b200 import frozen_io, synth
from tests import helpers as H


def test_coarse_snapshot_reads_the_reference_fixture():
    snap = frozen_io.read_coarse_snapshot(os.path.join(H.GOLDEN, "kat257"))
    meta, vals, rows, cols, rhs, ref, _, _ = H.load_kat257()
    assert snap.blocks == meta["coarse_block_nodes"] == 257
    assert np.array_equal(snap.rows, rows) and np.array_equal(snap.cols, cols)
    assert np.array_equal(snap.vals, vals) and np.array_equal(snap.rhs, rhs) and np.array_equal(snap.solution, ref)


def test_coarse_snapshot_round_trip_and_replay_inputs(tmp_path):
    snap = frozen_io.read_coarse_snapshot(os.path.join(H.GOLDEN, "kat257"))
    frozen_io.write_coarse_snapshot(str(tmp_path), snap)
    back = frozen_io.read_coarse_snapshot(str(tmp_path))
    for a in ("rows", "cols", "vals", "rhs", "solution"):
        assert np.array_equal(getattr(back, a), getattr(snap, a))
    assert back.metadata["coarse_unique_blocks"] == len(snap.rows)
    # the replay preparation matches the reference replay's (identity padding,
    # symmetric sorted unique neighbour lists, identity partition)
    k = frozen_io.coarse_replay_inputs(snap)
    old = H.kat257_padded()
    for a in ("vals", "rows", "cols", "rhs", "ref", "start", "num", "lst", "ident"):
        assert np.array_equal(np.asarray(k[a]), np.asarray(old[a])), a
    assert k["padded"] == old["padded"] and k["limit"] == old["limit"]


def test_frozen_system_round_trip(tmp_path):
    s = synth.config_system(0, scale=6)
    frozen_io.write_frozen(str(tmp_path), s.rows, s.cols, s.vals, s.b)
    assert sorted(os.listdir(tmp_path)) == sorted(frozen_io.FROZEN_FILES)
    f = frozen_io.read_frozen(str(tmp_path))
    assert f.block_rows == s.nb
    assert np.array_equal(f.rows, s.rows) and np.array_equal(f.cols, s.cols)
    assert np.array_equal(f.vals, s.vals) and np.array_equal(f.b, s.b)
    # raw layout: 72 bytes per block (Eigen::Matrix3d), 4 bytes per index
    assert os.path.getsize(tmp_path / "frozen_A_values.bin") == 72 * len(s.rows)
    assert os.path.getsize(tmp_path / "frozen_A_rows.bin") == 4 * len(s.rows)


def test_frozen_system_rejects_bad_indices(tmp_path):
    s = synth.config_system(0, scale=4)
    rows = s.rows.copy()
    rows[0] = s.nb  # out of range
    frozen_io.write_frozen(str(tmp_path), rows, s.cols, s.vals, s.b)
    try:
        frozen_io.read_frozen(str(tmp_path))
    except ValueError as e:
        assert "out of bounds" in str(e)
    else:
        raise AssertionError("accepted an out-of-range block index")
