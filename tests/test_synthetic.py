"""The seeded generators that stand in for the benchmark volumes (CPU, small sizes): determinism,
layout, and the rules each one states."""
import numpy as np

from brook_b200 import synthetic


def test_tube_volume_is_seeded_and_fortran_ordered():
    a = synthetic.tube_volume((40, 32, 24), objects=6, seed=3)
    b = synthetic.tube_volume((40, 32, 24), objects=6, seed=3)
    c = synthetic.tube_volume((40, 32, 24), objects=6, seed=4)
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)
    assert a.shape == (40, 32, 24) and a.dtype == np.uint32 and a.flags.f_contiguous
    assert set(np.unique(a)) <= set(range(7)) and (a > 0).any()
    assert synthetic.tube_volume((16, 16, 16), objects=2, seed=1, dtype=np.uint64).dtype == np.uint64


def test_dense_volume_cells_touch_only_through_background():
    v = synthetic.dense_volume((40, 36, 28), seeds=12, seed=5)
    assert v.dtype == np.uint64 and v.flags.f_contiguous
    ids = np.unique(v)
    assert ids[0] == 0 and 2 < len(ids) <= 13
    for axis in range(3):  # boundaries are eroded: no two different cells are face neighbours
        a = np.moveaxis(v, axis, 0)
        u, w = a[1:], a[:-1]
        assert not np.any((u != w) & (u != 0) & (w != 0))
    np.testing.assert_array_equal(v, synthetic.dense_volume((40, 36, 28), seeds=12, seed=5))


def test_arbor_walks_stay_within_their_step_count():
    rng = np.random.default_rng(0)
    centres = synthetic._walk(rng, (64, 64, 64), (32.0, 32.0, 32.0), 300, 0.5, limit=900)
    assert 0 < len(centres) <= 900  # a high branch probability would grow without the limit


def test_uneven_batch_and_requests_shapes():
    vols = synthetic.uneven_batch(count=3, edges=(16, 32), tubes=(2, 4), arbor_fraction=0.0)
    assert len(vols) == 3
    for v in vols:
        assert v.ndim == 3 and all(16 <= s <= 32 for s in v.shape) and v.dtype == np.uint32
    reqs = synthetic.serving_requests(4, rate=100.0, edges=(16, 24))
    times = [t for t, _ in reqs]
    assert times == sorted(times) and times[0] > 0
    assert {v.dtype for _, v in reqs} <= {np.dtype(np.uint32), np.dtype(np.uint64)}


def test_cell_volume_has_enclosed_nuclei_and_cavities():
    from scipy import ndimage

    v = synthetic.cell_volume((64, 64, 64), cells=8, seed=1)
    assert v.dtype == np.uint32 and v.flags.f_contiguous
    labels = set(np.unique(v).tolist()) - {0}
    assert labels == set(range(1, 17))  # 8 cells and their 8 nuclei
    for nucleus in range(9, 17):
        cell = nucleus - 8
        grown = ndimage.binary_dilation(v == nucleus)
        ring = np.unique(v[grown & (v != nucleus)])
        assert set(ring.tolist()) <= {0, cell}  # a nucleus touches only its own cell
    assert np.array_equal(synthetic.cell_volume((64, 64, 64), cells=8, seed=1), v)
