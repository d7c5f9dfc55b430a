"""Packed results on the host (no GPU): PackedSkeletons (the reference's src/brook/_packed.py) and
BatchedSkeletons (src/brook/batch.py:15-99), built from hand-made arrays."""
import numpy as np
import pytest

from brook_b200._packed import PackedSkeletons, Skeleton
from brook_b200.batch import BatchedSkeletons

ANISO = (4.0, 4.0, 40.0)


def packed(labels, sizes, seed):
    """Skeleton k: sizes[k] vertices on a chain (sizes[k] - 1 local edges)."""
    rng = np.random.default_rng(seed)
    v_off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    e_off = np.concatenate([[0], np.cumsum([max(s - 1, 0) for s in sizes])]).astype(np.int64)
    vertices = rng.random((int(v_off[-1]), 3)).astype(np.float32)
    edges = np.concatenate([np.stack([np.arange(s - 1), np.arange(1, s)], 1) for s in sizes] or [np.zeros((0, 2))])
    radii = rng.random(int(v_off[-1])).astype(np.float32)
    return PackedSkeletons(np.asarray(labels, np.int64), v_off, e_off, vertices, edges.astype(np.uint32), radii, ANISO)


def test_to_skeletons_slices_each_skeleton():
    p = packed([7, 3], [4, 2], seed=1)
    out = p.to_skeletons()
    assert sorted(out) == [3, 7]
    s7, s3 = out[7], out[3]
    assert isinstance(s7, Skeleton) and s7.id == 7
    np.testing.assert_array_equal(s7.vertices, p.vertices[0:4])
    np.testing.assert_array_equal(s3.vertices, p.vertices[4:6])
    np.testing.assert_array_equal(s7.edges, [[0, 1], [1, 2], [2, 3]])
    np.testing.assert_array_equal(s3.edges, [[0, 1]])
    np.testing.assert_array_equal(s3.radii, p.radii[4:6])
    np.testing.assert_array_equal(s7.transform, [[4, 0, 0, 0], [0, 4, 0, 0], [0, 0, 40, 0]])
    assert len(p) == 2 and not p.on_device and p.to_host() is p


def test_empty_packed():
    e = PackedSkeletons.empty(ANISO)
    assert len(e) == 0 and e.to_skeletons() == {}
    assert e.v_off.tolist() == [0] and e.e_off.tolist() == [0]


def test_concatenate_and_index_round_trip():
    parts = [packed([5, 9], [3, 5], seed=2), PackedSkeletons.empty(ANISO), packed([5], [2], seed=3)]
    b = BatchedSkeletons.concatenate(parts, ANISO)
    assert len(b) == 3
    assert b.s_off.tolist() == [0, 2, 2, 3]
    assert b.sample.tolist() == [0, 0, 2]
    assert b.labels.tolist() == [5, 9, 5]  # labels are per sample: they may repeat across samples
    assert b.v_off.tolist() == [0, 3, 8, 10] and b.e_off.tolist() == [0, 2, 6, 7]
    for i, part in enumerate(parts):
        got = b[i]
        np.testing.assert_array_equal(got.labels, part.labels)
        np.testing.assert_array_equal(got.v_off, part.v_off)
        np.testing.assert_array_equal(got.e_off, part.e_off)
        np.testing.assert_array_equal(got.vertices, part.vertices.reshape(-1, 3))
        np.testing.assert_array_equal(got.edges, part.edges.reshape(-1, 2))
        np.testing.assert_array_equal(got.radii, part.radii)
    np.testing.assert_array_equal(b[-1].vertices, b[2].vertices)
    with pytest.raises(IndexError):
        b[3]
    dicts = b.to_skeletons()
    assert [sorted(d) for d in dicts] == [[5, 9], [], [5]]
    np.testing.assert_array_equal(dicts[2][5].vertices, parts[2].vertices)


def test_concatenate_nothing():
    b = BatchedSkeletons.concatenate([], ANISO)
    assert len(b) == 0 and b.s_off.tolist() == [0]
    assert b.vertices.shape == (0, 3) and b.edges.shape == (0, 2)
