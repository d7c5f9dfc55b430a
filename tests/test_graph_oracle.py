"""The voxel-graph oracle (oracle/graph.cpp: graph components and the graph-aware EDT) against the
reference's own known answers, hand-derived half-voxel distances, and invariants on seeded
volumes (CPU only)."""
import numpy as np
import pytest
from scipy import ndimage

from oracle import graph as og

OPEN = np.uint32((1 << 26) - 1)


def test_reference_known_answers():
    # cpp/tests/c_smoke.c:8-13, 36-52 of the reference: eight voxels in a row, an all-zero graph
    labels = np.array([1, 1, 0, 0, 0, 0, 2, 2], np.uint8)
    ids, mapping, roots, keys = og.graph_components(labels, np.zeros(8, np.uint32))
    np.testing.assert_array_equal(ids.ravel(), [1, 2, 0, 0, 0, 0, 3, 4])
    assert len(roots) == 4 and mapping[3] == 2 and mapping[4] == 2 and roots[2] == 6 and roots[3] == 7
    np.testing.assert_array_equal(keys, [0, 1, 2, 7, 8])  # ranks among all eight one-voxel components
    gd = og.graph_edt(labels, np.zeros(8, np.uint32))
    np.testing.assert_array_equal(gd.ravel(), np.where(labels > 0, 0.5, 0.0).astype(np.float32))


def test_half_voxel_interfaces():
    # a voxel's own +x face interface sits half a voxel after it and is blocked by its graph's bit
    # 0; the background before a voxel is half a voxel nearer than the background after it
    line = np.array([0, 1, 1, 1, 0])
    np.testing.assert_array_equal(og.graph_edt(line, np.full(5, OPEN)).ravel(), [0, 0.5, 1.5, 1.0, 0])
    cut = np.full(5, OPEN)
    cut[2] &= ~np.uint32(1)
    np.testing.assert_array_equal(og.graph_edt(line, cut).ravel(), [0, 0.5, 0.5, 0.5, 0])
    np.testing.assert_array_equal(og.graph_edt(line, np.full(5, OPEN), anisotropy=(4, 1, 1)).ravel(),
                                  [0, 2, 6, 4, 0])
    # a black border closes the last doubled slice of every axis and the space before the first:
    # in a full 3x3x3 block only the centre is more than half a voxel from it
    full = np.ones((3, 3, 3), np.uint32)
    border = og.graph_edt(full, np.full(full.shape, OPEN), black_border=True)
    expected = np.full(full.shape, 0.5, np.float32)
    expected[1, 1, 1] = 1.5
    np.testing.assert_array_equal(border, expected)
    assert np.all(np.isinf(og.graph_edt(full, np.full(full.shape, OPEN))))  # no zero anywhere


def _components_by_label(labels):
    """26-connected components of each label (background included) in order of their lowest
    voxel in Fortran order: (ids with background 0, mapping, roots, keys)."""
    flat_index = np.arange(labels.size).reshape(labels.shape, order="F")
    comps = []
    for value in np.unique(labels):
        lab, count = ndimage.label(labels == value, structure=np.ones((3, 3, 3)))
        for c in range(1, count + 1):
            comps.append((int(flat_index[lab == c].min()), int(value), lab == c))
    comps.sort(key=lambda t: t[0])
    ids = np.zeros(labels.shape, np.uint32)
    mapping, roots, keys = [0], [], [0]
    for rank, (low, value, where) in enumerate(comps, start=1):
        if value == 0:
            continue
        ids[where] = len(roots) + 1
        mapping.append(value)
        roots.append(low)
        keys.append(rank)
    return ids, np.array(mapping), np.array(roots), np.array(keys)


@pytest.mark.parametrize("seed", range(6))
def test_label_graph_gives_the_labels_components(seed):
    rng = np.random.default_rng(seed)
    shape = tuple(int(s) for s in rng.integers(3, 9, 3))
    labels = rng.integers(0, 4, shape).astype(np.uint16)
    labels[rng.random(shape) < 0.4] = 0
    labels = np.asfortranarray(labels)
    got = og.graph_components(labels, og.label_graph(labels))
    exp = _components_by_label(labels)
    for a, b, name in zip(got, exp, ("ids", "mapping", "roots", "keys")):
        np.testing.assert_array_equal(np.asarray(a), np.asarray(b), err_msg=name)


def test_cut_splits_and_spanning_component_mapping():
    # two bars of one label touching along a face: the labels' graph without the steps across the
    # contact (the reference's _graph_cases, tests/python/test_package.py:1255-1283) gives two
    # components, the labels alone one
    bars = np.zeros((12, 12, 8), np.uint32)
    bars[2:10, 2:6, 2:6] = 1
    bars[2:10, 6:10, 2:6] = 1
    side = np.zeros(bars.shape, bool)
    side[:, 6:, :] = True
    graph = og.label_graph(bars)
    for bit, (dx, dy, dz) in enumerate(og.STEPS):
        src = tuple(slice(max(0, -d), bars.shape[a] - max(0, d)) for a, d in enumerate((dx, dy, dz)))
        dst = tuple(slice(max(0, d), bars.shape[a] - max(0, -d)) for a, d in enumerate((dx, dy, dz)))
        graph[src] &= ~((side[src] != side[dst]).astype(np.uint32) << np.uint32(bit))
    ids, mapping, roots, _ = og.graph_components(bars, graph)
    assert len(roots) == 2 and set(np.unique(ids)) == {0, 1, 2}
    assert np.all(ids[side & (bars > 0)] == 2) and np.all(ids[~side & (bars > 0)] == 1)
    assert len(og.graph_components(bars, og.label_graph(bars))[2]) == 1
    # labels 5 and 9 that an all-steps graph joins (the reference's _spanning_labels,
    # tests/python/test_package.py:1446-1455): one component, whose last run of voxels in
    # Fortran order starts in label 5
    labels = np.zeros((12, 6, 10), np.uint32)
    labels[1:6, 1:5, 5:9] = 5
    labels[6:11, 1:5, 1:9] = 9
    ids, mapping, roots, keys = og.graph_components(np.asfortranarray(labels), np.full(labels.shape, OPEN))
    assert list(mapping) == [0, 5] and list(keys) == [0, 1]
    assert roots[0] == np.ravel_multi_index((6, 1, 1), labels.shape, order="F")


def test_compact_2d_graph():
    """A uint8 graph of a 2D volume holds the 3D bits 0-3 and 6-9 in bits 0-7."""
    rng = np.random.default_rng(3)
    labels = rng.integers(0, 3, (9, 7, 1)).astype(np.uint8)
    wide = np.asfortranarray(og.label_graph(labels) & rng.integers(0, 1 << 26, labels.shape, dtype=np.uint32))
    compact = ((wide & 0xF) | ((wide >> 2) & 0xF0)).astype(np.uint8)
    for a, b in zip(og.graph_components(labels, wide), og.graph_components(labels, np.asfortranarray(compact))):
        np.testing.assert_array_equal(a, b)


def test_refusals():
    with pytest.raises(ValueError):
        og.graph_components(np.ones(4, np.uint8), np.zeros(3, np.uint32))
    with pytest.raises(ValueError):
        og.graph_edt(np.ones(4, np.uint8), np.zeros(4, np.uint16))
    with pytest.raises(ValueError):
        og.graph_edt(np.ones(4, np.uint8), np.zeros(4, np.uint32), anisotropy=(0, 1, 1))
