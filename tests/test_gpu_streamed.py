"""The out-of-core path (brook_skeletonize_streamed / brook_connected_components_streamed): small
device budgets force many slabs and many crop batches; the skeletons must equal the in-core call's
and the oracle's bit for bit (labels and their order, offsets, vertices, edges, radii), and the
streamed components the in-core components."""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from test_gpu_parity import CFG0_PARAMS, assert_same

pytestmark = pytest.mark.gpu


def streamed(labels, budget, **options):
    """skeletonize through brook_skeletonize_streamed with an explicit budget (bytes)."""
    import brook_b200
    from brook_b200 import _intake, _native

    keep = _intake.format_labels(labels)
    params = _intake.teasar(options.pop("teasar_params", brook_b200.DEFAULT_TEASAR_PARAMS))
    aniso = tuple(float(a) for a in np.asarray(options.pop("anisotropy", (1, 1, 1)), np.float32))
    ids = options.pop("object_ids", None)
    before = [tuple(int(c) for c in p) for p in options.pop("extra_targets_before", ())]
    after = [tuple(int(c) for c in p) for p in options.pop("extra_targets_after", ())]
    out = _intake._run_streamed(_native.host_volume(keep), params, aniso, ids, options.pop("dust_threshold", 1000),
                                options.pop("fix_branching", True), options.pop("fix_borders", True), before, after,
                                0, budget=budget)
    assert not options, options
    return out


def assert_packed_equal(a, b, what=""):
    for key in ("labels", "v_off", "e_off", "edges"):
        np.testing.assert_array_equal(np.asarray(getattr(a, key)), np.asarray(getattr(b, key)), err_msg=f"{what} {key}")
    np.testing.assert_array_equal(np.asarray(a.vertices).view(np.uint32), np.asarray(b.vertices).view(np.uint32),
                                  err_msg=f"{what} vertices")
    np.testing.assert_array_equal(np.asarray(a.radii).view(np.uint32), np.asarray(b.radii).view(np.uint32),
                                  err_msg=f"{what} radii")


@pytest.mark.parametrize("budget", [1 << 20, 4 << 20, 256 << 20])
def test_tubes_streamed_equal_in_core_and_oracle(gpu, budget):
    import brook_b200
    from brook_b200 import _native, synthetic

    labels = synthetic.tube_volume((96, 80, 64), objects=14, seed=3, arbor_fraction=0.2)
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(8, 8, 40), dust_threshold=50)
    got = streamed(labels, budget, **opts)
    stats = _native.stats()
    assert got.labels.size > 5
    assert_packed_equal(got, brook_b200.skeletonize(labels, output="packed", **opts), f"budget {budget}")
    assert_same(got, oracle.skeletonize(labels, threads=8, **opts), f"oracle, budget {budget}")
    if budget == 1 << 20:
        assert stats["streamed_slabs"] > 4 and stats["streamed_batches"] > 2


def test_dense_cells_with_border_targets(gpu):
    """Components touching every face (border targets from the whole volume's faces), uint64, C order."""
    import brook_b200
    from brook_b200 import synthetic

    labels = np.ascontiguousarray(synthetic.dense_volume((80, 72, 48), seeds=30, seed=2))
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100)
    got = streamed(labels, 2 << 20, **opts)
    assert_packed_equal(got, brook_b200.skeletonize(labels, output="packed", **opts), "dense")


def test_black_border_split_labels_targets_and_object_ids(gpu):
    import brook_b200

    full = np.ones((20, 14, 12), np.uint16)
    opts = dict(dust_threshold=0, anisotropy=(2, 3, 4))
    assert_packed_equal(streamed(full, 1 << 16, **opts), brook_b200.skeletonize(full, output="packed", **opts),
                        "one object filling the volume")
    two = np.zeros((40, 30, 32), np.uint32)
    two[2:16, 2:5, 2:5] = 9
    two[24:38, 20:24, 20:30] = 9      # a second component of label 9, in a later slab
    two[2:36, 10:13, 12:30] = 5
    two[30:34, 2:28, 3:6] = 7
    opts = dict(dust_threshold=0, anisotropy=(1, 1, 1), extra_targets_before=[(3, 3, 3)],
                extra_targets_after=[(-3, 11, 20), (31, 5, 4)])
    assert_packed_equal(streamed(two, 1 << 15, **opts), brook_b200.skeletonize(two, output="packed", **opts),
                        "split label, targets")
    opts = dict(dust_threshold=0, object_ids=[9, 7])
    got = streamed(two, 1 << 15, **opts)
    assert sorted(got.labels.tolist()) == [7, 9]
    assert_packed_equal(got, brook_b200.skeletonize(two, output="packed", **opts), "object_ids")


def test_somata_streamed(gpu):
    """Soma candidates and somata run in their crops as in-core (voids, DBF refresh, soma root)."""
    import brook_b200
    from brook_b200 import synthetic
    from test_oracle_golden import SOMA_PARAMS

    labels = synthetic.tube_volume((96, 88, 72), objects=8, seed=4, radius=(1.5, 3.0)).astype(np.uint32)
    grid = np.indices(labels.shape)
    for label, centre, radius in ((21, (30, 30, 30), 11), (22, (70, 60, 40), 9), (23, (60, 20, 55), 6)):
        labels[sum((g - c) ** 2 for g, c in zip(grid, centre)) <= radius ** 2] = label
    labels[26:34, 27:33, 28:32] = 0
    labels[29:31, 29:31, 29:31] = 30
    labels[30, 0:30, 30] = 21
    params = dict(SOMA_PARAMS, soma_detection_threshold=5.5, soma_acceptance_threshold=8.5)
    opts = dict(teasar_params=params, anisotropy=(1, 1, 1.25), dust_threshold=5)
    got = streamed(np.asfortranarray(labels), 2 << 20, **opts)
    assert_packed_equal(got, brook_b200.skeletonize(np.asfortranarray(labels), output="packed", **opts), "somata")


def test_streamed_components_equal_in_core(gpu):
    from brook_b200 import _native, synthetic

    lib, ctx = _native.load(), _native.context(0)
    labels = np.asfortranarray(synthetic.dense_volume((64, 48, 40), seeds=25, seed=7, dtype=np.uint32))
    vol = _native.host_volume(labels)
    hc = ctypes.c_void_p()
    _native.check(lib.brook_connected_components_streamed(ctx, ctypes.byref(vol), 1 << 16, ctypes.byref(hc)))
    view, mapping, roots, count = _native.Volume(), ctypes.POINTER(ctypes.c_int64)(), ctypes.POINTER(ctypes.c_int64)(), \
        ctypes.c_size_t()
    _native.check(lib.brook_host_components_view(hc, ctypes.byref(view), ctypes.byref(mapping), ctypes.byref(roots),
                                                 ctypes.byref(count)))
    dt = {0: np.uint8, 1: np.uint16, 2: np.uint32}[view.dtype]
    n = labels.size
    got_ids = np.ctypeslib.as_array(ctypes.cast(view.data, ctypes.POINTER(ctypes.c_uint8)), (n * np.dtype(dt).itemsize,))
    got_ids = got_ids.view(dt).reshape(labels.shape, order="F").copy()
    got_map = np.ctypeslib.as_array(mapping, (count.value + 1,)).copy()
    got_roots = np.ctypeslib.as_array(roots, (count.value,)).copy()
    lib.brook_host_components_destroy(hc)
    assert _native.stats()["streamed_slabs"] > 4
    cc = ctypes.c_void_p()
    _native.check(lib.brook_connected_components(ctx, ctypes.byref(vol), ctypes.byref(cc)))
    cview, cmap, croots, ccount = _native.Volume(), ctypes.POINTER(ctypes.c_int64)(), ctypes.POINTER(ctypes.c_int64)(), \
        ctypes.c_size_t()
    _native.check(lib.brook_components_view(cc, ctypes.byref(cview), ctypes.byref(cmap), ctypes.byref(croots),
                                            ctypes.byref(ccount)))
    assert ccount.value == count.value
    exp = np.zeros(labels.shape, dt, order="F")
    _native.check(lib.brook_components_copy_to_host(cc, exp.ctypes.data, exp.nbytes))
    np.testing.assert_array_equal(got_ids, exp)
    np.testing.assert_array_equal(got_map, np.ctypeslib.as_array(cmap, (ccount.value + 1,)))
    np.testing.assert_array_equal(got_roots, np.ctypeslib.as_array(croots, (ccount.value,)))
    lib.brook_components_destroy(cc)


def test_streaming_selection_and_refusals(gpu, monkeypatch):
    import torch

    import brook_b200
    from brook_b200 import _native, synthetic

    labels = synthetic.tube_volume((48, 40, 32), objects=4, seed=1)
    opts = dict(teasar_params=CFG0_PARAMS, dust_threshold=10)
    monkeypatch.setenv("BROOK_STREAM_BUDGET_MB", "1")
    a = brook_b200.skeletonize(labels, streaming=True, output="packed", **opts)
    assert _native.stats()["streamed_slabs"] > 1
    assert_packed_equal(a, brook_b200.skeletonize(labels, streaming=False, output="packed", **opts), "streaming=True")
    monkeypatch.setenv("BROOK_STREAMING", "1")
    b = brook_b200.skeletonize(labels, output="packed", **opts)
    assert_packed_equal(a, b, "BROOK_STREAMING=1")
    with pytest.raises(NotImplementedError):
        brook_b200.skeletonize(labels, streaming=True, fill_holes=True, **opts)
    with pytest.raises(NotImplementedError):
        brook_b200.skeletonize(torch.from_numpy(np.asfortranarray(labels)).cuda(), streaming=True, **opts)
    d = brook_b200.skeletonize(labels, streaming=True, output="packed_device", **opts)
    assert d.on_device
    assert_packed_equal(d.to_host(), a, "device output")


@pytest.mark.parametrize("black_border", [0, 1])
def test_edt_streamed_equals_in_core(gpu, black_border):
    """brook_edt_streamed (x/y passes by z-slabs, the z pass by column tiles) gives brook_edt's
    field bit for bit, C-ordered uint16 input, a budget of a few planes."""
    from brook_b200 import _native, synthetic

    lib, ctx = _native.load(), _native.context(0)
    labels = np.ascontiguousarray(synthetic.dense_volume((72, 56, 48), seeds=20, seed=3, dtype=np.uint16))
    aniso = (ctypes.c_float * 3)(4.0, 4.0, 40.0)
    vol = _native.host_volume(labels)
    out = np.zeros(labels.shape, np.float32, order="F")
    _native.check(lib.brook_edt_streamed(ctx, ctypes.byref(vol), aniso, black_border, 1 << 18, out.ctypes.data,
                                         out.nbytes))
    assert _native.stats()["launches"] > 10
    arr = ctypes.c_void_p()
    _native.check(lib.brook_edt(ctx, ctypes.byref(vol), aniso, black_border, ctypes.byref(arr)))
    exp = np.zeros(labels.shape, np.float32, order="F")
    _native.check(lib.brook_array_copy_to_host(arr, exp.ctypes.data, exp.nbytes))
    lib.brook_array_destroy(arr)
    np.testing.assert_array_equal(out.view(np.uint32), exp.view(np.uint32))
    small = np.zeros(4, np.float32)
    with pytest.raises(_native.BrookError):
        _native.check(lib.brook_edt_streamed(ctx, ctypes.byref(vol), aniso, black_border, 0, small.ctypes.data,
                                             small.nbytes))
