"""Parity of the CUDA path (through the C ABI) with the CPU oracle and the reference's known answers.

Integer/index results (vertices, edges, labels, offsets) must be identical; radii are compared
bit-exactly too (both sides compute the same float32 EDT)."""
import ctypes
import json
import os

import numpy as np
import pytest

import shapes
from oracle import oracle

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "join_digests.json")))
CFG0_PARAMS = dict(scale=1.5, const=300, pdrf_scale=100000, pdrf_exponent=4)


def bk():
    import brook_b200

    return brook_b200


def assert_same(packed, expected, what=""):
    """packed (brook_b200 PackedSkeletons) equals the oracle's packed result exactly."""
    e = expected.packed()
    np.testing.assert_array_equal(packed.labels, e["labels"], err_msg=f"labels {what}")
    np.testing.assert_array_equal(packed.v_off, e["vertex_offsets"], err_msg=f"vertex offsets {what}")
    np.testing.assert_array_equal(packed.e_off, e["edge_offsets"], err_msg=f"edge offsets {what}")
    np.testing.assert_array_equal(packed.vertices, e["vertices"], err_msg=f"vertices {what}")
    np.testing.assert_array_equal(packed.edges, e["edges"], err_msg=f"edges {what}")
    np.testing.assert_array_equal(packed.radii.view(np.uint32), e["radii"].view(np.uint32), err_msg=f"radii {what}")


def run_both(labels, threads=8, **options):
    got = bk().skeletonize(labels, output="packed", **options)
    exp = oracle.skeletonize(labels, threads=threads, **options)
    return got, exp


@pytest.mark.parametrize("case", sorted(shapes.CASES))
@pytest.mark.parametrize("layout", [np.ascontiguousarray, np.asfortranarray])
def test_join_digests(gpu, case, layout):
    make, extra = shapes.CASES[case]
    opts = dict(shapes.JOIN_OPTIONS, **extra)
    result = bk().skeletonize(layout(make()), output="packed", **opts)
    summary = shapes.summary({int(l): (s.vertices, s.edges, s.radii) for l, s in result.to_skeletons().items()})
    assert summary == {int(k): v for k, v in GOLDEN[case].items()}


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_tubes_match_oracle(gpu, seed):
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((64, 64, 64), objects=8, seed=seed)
    got, exp = run_both(labels, teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100)
    assert len(got) > 0
    assert_same(got, exp, f"seed {seed}")


def test_cfg0_full_size_matches_oracle(gpu):
    """The 128^3 uint32 volume of 20 random-walk tubes (seed 0), anisotropy (16,16,40)."""
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((128, 128, 128), objects=20, seed=0)
    got, exp = run_both(labels, teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100)
    assert len(got) == 20
    assert_same(got, exp, "cfg0")


@pytest.mark.parametrize("cluster_voxels", ["1", "1000000000"])
def test_cluster_and_lone_cta_paths_match_oracle(gpu, monkeypatch, cluster_voxels):
    """Every object on a thread-block cluster ("1"), or every object on one CTA: the same skeletons."""
    from brook_b200 import synthetic

    monkeypatch.setenv("BROOK_B200_PREPARE_CLUSTER_VOXELS", cluster_voxels)
    monkeypatch.setenv("BROOK_B200_TRACE_CLUSTER_VOXELS", cluster_voxels)
    labels = synthetic.tube_volume((96, 96, 96), objects=12, seed=3)
    got, exp = run_both(labels, teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100)
    assert len(got) == 12
    assert_same(got, exp, f"cluster threshold {cluster_voxels}")


def test_wide_target_order_key_matches_oracle(gpu, monkeypatch):
    """The (32, 64)-bit target-order sort key, used when object, DAF and position need > 64 bits."""
    from brook_b200 import synthetic

    monkeypatch.setenv("BROOK_B200_WIDE_ORDER_KEY", "1")
    labels = synthetic.tube_volume((96, 96, 96), objects=12, seed=3)
    got, exp = run_both(labels, teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100)
    assert len(got) == 12
    assert_same(got, exp, "wide order key")


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.uint64, np.int32, np.int64])
def test_dtypes(gpu, dtype):
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((48, 40, 36), objects=6, seed=7, radius=(1.5, 4.0)).astype(dtype)
    got, exp = run_both(labels, teasar_params=dict(scale=1.0, const=2.0), anisotropy=(4, 4, 4), dust_threshold=20)
    assert_same(got, exp, str(np.dtype(dtype)))


@pytest.mark.parametrize("aniso", [(1, 1, 1), (4, 4, 4), (8, 8, 40), (16, 16, 40)])
def test_anisotropies(gpu, aniso):
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((40, 56, 48), objects=5, seed=3, radius=(1.5, 5.0))
    got, exp = run_both(labels, teasar_params=CFG0_PARAMS, anisotropy=aniso, dust_threshold=50)
    assert_same(got, exp, str(aniso))


def test_dense_cells_match_oracle(gpu):
    """Voronoi cells cut by tubes (the dense-segmentation generator) at 128^3, uint64 ids."""
    from brook_b200 import synthetic

    labels = synthetic.dense_volume((128, 128, 128), seeds=40, seed=5)
    got, exp = run_both(labels, teasar_params=CFG0_PARAMS, anisotropy=(8, 8, 40), dust_threshold=100)
    assert len(got) > 10
    assert_same(got, exp, "dense")


def test_empty_and_dust(gpu):
    b = bk()
    assert b.skeletonize(np.zeros((0, 4, 4), np.uint32), dust_threshold=0) == {}
    assert b.skeletonize(np.zeros((16, 16, 16), np.uint32), dust_threshold=0) == {}
    assert b.skeletonize(np.ones((4, 4, 4), np.uint32), dust_threshold=64) == {}


def test_tiny_objects(gpu):
    v = np.zeros((8, 8, 8), np.uint32)
    v[1, 1, 1] = 3
    v[5, 5, 5] = 4
    v[5, 5, 6] = 4
    got, exp = run_both(v, dust_threshold=0, anisotropy=(1, 1, 1))
    assert_same(got, exp, "tiny")
    assert list(got.labels) == [4]


def test_black_border(gpu):
    """One object filling the whole volume: the volume edge counts as background."""
    full = np.ones((12, 10, 9), np.uint16)
    got, exp = run_both(full, dust_threshold=0, anisotropy=(2, 3, 4))
    assert_same(got, exp, "full")


def test_flat_and_line(gpu):
    flat = shapes.sine_band(6.0, 60.0, 1.6, axis=2)
    got, exp = run_both(flat, dust_threshold=0, anisotropy=(4, 4, 4), teasar_params=dict(scale=1.0, const=2.0))
    assert_same(got, exp, "flat")
    line = np.zeros((30, 1, 1), np.uint8)
    line[3:27] = 1
    got, exp = run_both(line, dust_threshold=0)
    assert_same(got, exp, "line")


def test_split_label_and_object_ids(gpu):
    """Two components of one label merge into one skeleton; object_ids keeps the listed labels."""
    two = np.zeros((20, 20, 20), np.uint32)
    two[2:8, 2:4, 2:4] = 9
    two[12:19, 14:16, 10:12] = 9
    two[2:18, 10:12, 16:18] = 5
    got, exp = run_both(two, dust_threshold=0, anisotropy=(1, 1, 1))
    assert_same(got, exp, "merge")
    only = bk().skeletonize(two, dust_threshold=0, object_ids=[5], output="packed")
    assert list(only.labels) == [5]


def test_fix_borders_off(gpu):
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((64, 64, 64), objects=8, seed=11)
    got, exp = run_both(labels, teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100,
                        fix_borders=False)
    assert_same(got, exp, "no borders")


def test_max_paths(gpu):
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((64, 64, 64), objects=6, seed=12)
    params = dict(CFG0_PARAMS, max_paths=3)
    got, exp = run_both(labels, teasar_params=params, anisotropy=(16, 16, 40), dust_threshold=100)
    assert_same(got, exp, "max_paths")


def test_device_input_and_layouts(gpu):
    import torch
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((48, 40, 36), objects=5, seed=21)
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=50)
    exp = oracle.skeletonize(labels, **opts)
    for host in (np.asfortranarray(labels), np.ascontiguousarray(labels), labels[:, :, :].transpose(0, 1, 2)):
        assert_same(bk().skeletonize(host, output="packed", **opts), exp, "host layout")
    # device tensors: Fortran-ordered (read in place) and C-ordered (gathered on the device)
    t_c = torch.from_numpy(np.ascontiguousarray(labels)).cuda()
    assert_same(bk().skeletonize(t_c, output="packed", **opts), exp, "device C")
    t_f = torch.from_numpy(np.ascontiguousarray(labels.transpose(2, 1, 0))).cuda().permute(2, 1, 0)
    assert_same(bk().skeletonize(t_f, output="packed", **opts), exp, "device F")


def test_batch_identity(gpu):
    """skeletonize_batch(samples)[i] == skeletonize(samples[i]) for uneven shapes and dtypes."""
    from brook_b200 import synthetic

    samples = [synthetic.tube_volume((40, 52, 33), objects=4, seed=31),
               synthetic.tube_volume((64, 30, 45), objects=6, seed=32).astype(np.uint16),
               np.zeros((10, 10, 10), np.uint32),
               synthetic.tube_volume((33, 33, 70), objects=3, seed=33).astype(np.uint64)]
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(4, 4, 4), dust_threshold=50)
    batch = bk().skeletonize_batch(samples, output="packed", **opts)
    assert len(batch) == len(samples)
    for i, s in enumerate(samples):
        assert_same(batch[i], oracle.skeletonize(s, **opts), f"sample {i}")


def test_c_abi_known_answers(gpu):
    """c_smoke.c:7-61 of the reference: components and EDT of {1,1,0,0,0,0,2,2}."""
    from brook_b200 import _native as n

    lib = n.lib
    labels = np.array([1, 1, 0, 0, 0, 0, 2, 2], np.uint8).reshape(8, 1, 1, order="F")
    vol = n.host_volume(labels)
    ctx = n.context(0)
    cc = ctypes.c_void_p()
    n.check(lib.brook_connected_components(ctx, ctypes.byref(vol), ctypes.byref(cc)))
    view = n.Volume()
    mapping = ctypes.POINTER(ctypes.c_int64)()
    roots = ctypes.POINTER(ctypes.c_int64)()
    count = ctypes.c_size_t()
    n.check(lib.brook_components_view(cc, ctypes.byref(view), ctypes.byref(mapping), ctypes.byref(roots),
                                      ctypes.byref(count)))
    assert count.value == 2 and mapping[1] == 1 and mapping[2] == 2 and roots[0] == 0 and roots[1] == 6
    out = np.zeros(8, np.uint8)
    n.check(lib.brook_components_copy_to_host(cc, out.ctypes.data, out.nbytes))
    assert out.tolist() == labels.ravel().tolist()
    lib.brook_components_destroy(cc)
    aniso = (ctypes.c_float * 3)(1, 1, 1)
    arr = ctypes.c_void_p()
    n.check(lib.brook_edt(ctx, ctypes.byref(vol), aniso, 0, ctypes.byref(arr)))
    d = np.zeros(8, np.float32)
    n.check(lib.brook_array_copy_to_host(arr, d.ctypes.data, d.nbytes))
    lib.brook_array_destroy(arr)
    assert d[0] == 2 and d[1] == 1 and d[2] == 0 and d[6] == 1 and d[7] == 2
    # errors map to status codes with a message
    bad = n.host_volume(labels)
    bad.abi_version = 99
    assert lib.brook_connected_components(ctx, ctypes.byref(bad), ctypes.byref(cc)) == n.INVALID_ARGUMENT
    assert lib.brook_last_error()


def _components_by_first_voxel(labels):
    """26-connected components of every label (scipy), numbered 1..K by ascending first voxel in
    Fortran order: the canonical numbering of brook.h:169-177."""
    from scipy import ndimage

    shape = labels.shape
    comps = []
    for value in np.unique(labels):
        if value == 0:
            continue
        lab, count = ndimage.label(labels == value, structure=np.ones((3, 3, 3), bool))
        flat = lab.ravel(order="F")
        idx = np.nonzero(flat)[0]
        first = np.full(count + 1, flat.size, np.int64)
        np.minimum.at(first, flat[idx], idx)
        for c in range(1, count + 1):
            comps.append((int(first[c]), (lab == c), int(value)))
    comps.sort(key=lambda t: t[0])
    ids = np.zeros(shape, np.int64)
    for k, (_, where, _) in enumerate(comps, start=1):
        ids[where] = k
    return ids, [t[0] for t in comps], [t[2] for t in comps]


@pytest.mark.parametrize("pair_capacity", [None, "0", "5"])
@pytest.mark.parametrize("shape,blob", [((70, 45, 37), 3), ((33, 9, 17), 1), ((128, 16, 24), 6), ((5, 300, 4), 2), ((40, 24, 20), 0)])
def test_connected_components_match_scipy(gpu, monkeypatch, shape, blob, pair_capacity):
    """Component ids, roots and labels of blobby random labels with noise, on sizes that are not
    multiples of the 32x8x8 union tiles, against scipy's 26-connected labelling; also with the
    list of cross-tile pairs overflowing (capacity 0 or 5), where the face scan takes over."""
    from scipy import ndimage
    from brook_b200 import _native as n

    if pair_capacity is not None:
        monkeypatch.setenv("BROOK_B200_TEST_PAIR_CAPACITY", pair_capacity)

    rng = np.random.default_rng(sum(shape) + blob)
    field = ndimage.gaussian_filter(rng.random((5,) + shape), sigma=(0, blob, blob, blob))
    labels = (np.argmax(field, axis=0) + 1).astype(np.uint64) * 1000003
    labels[rng.random(shape) < 0.15] = 0
    labels = np.asfortranarray(labels)
    expected, roots_expected, values = _components_by_first_voxel(labels)
    lib = n.lib
    ctx = n.context(0)
    vol = n.host_volume(labels)
    cc = ctypes.c_void_p()
    n.check(lib.brook_connected_components(ctx, ctypes.byref(vol), ctypes.byref(cc)))
    view = n.Volume()
    mapping = ctypes.POINTER(ctypes.c_int64)()
    roots = ctypes.POINTER(ctypes.c_int64)()
    count = ctypes.c_size_t()
    n.check(lib.brook_components_view(cc, ctypes.byref(view), ctypes.byref(mapping), ctypes.byref(roots),
                                      ctypes.byref(count)))
    k = count.value
    assert k == len(roots_expected)
    dtype = np.uint8 if k <= 0xFF else np.uint16 if k <= 0xFFFF else np.uint32
    out = np.zeros(labels.size, dtype)
    n.check(lib.brook_components_copy_to_host(cc, out.ctypes.data, out.nbytes))
    got_roots = [roots[i] for i in range(k)]
    got_values = [mapping[i + 1] for i in range(k)]
    lib.brook_components_destroy(cc)  # the view's arrays end with the handle
    np.testing.assert_array_equal(out.reshape(shape, order="F").astype(np.int64), expected)
    assert got_roots == roots_expected
    assert got_values == values


def test_threads_with_other_x_extents_do_not_race(gpu):
    """Threads, each with its own context, run EDTs of different x extents at once (one above the
    48 KiB default shared-memory limit of the x pass): the limit is a process-wide attribute of the
    kernel, so no call may lower it for another's launch."""
    import threading
    from brook_b200 import _native as n

    errors = []

    def work(sx):
        try:
            labels = np.asfortranarray(np.ones((sx, 6, 5), np.uint32))
            labels[sx // 2] = 2
            ctx = n.context(0)
            for _ in range(40):
                vol = n.host_volume(labels)
                arr = ctypes.c_void_p()
                n.check(n.lib.brook_edt(ctx, ctypes.byref(vol), (ctypes.c_float * 3)(1, 1, 1), 0, ctypes.byref(arr)))
                n.lib.brook_array_destroy(arr)
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append(e)

    threads = [threading.Thread(target=work, args=(sx,)) for sx in (40, 700, 3500)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors


def test_c_abi_device_output(gpu):
    """BROOK_DEVICE_OUTPUT (brook.h:96-102, 232-233): the device view and array handles hold the
    same skeletons as the host route; get_view copies a device result to the host; a host result
    has no device view."""
    from brook_b200 import _native as n
    from brook_b200 import _intake, synthetic

    labels = np.asfortranarray(synthetic.tube_volume((64, 64, 64), objects=8, seed=5))
    vol = n.host_volume(labels)
    ctx = n.context(0)
    opts = n.options(_intake.teasar(CFG0_PARAMS), (16, 16, 40), 100, True, True)
    host = ctypes.c_void_p()
    n.check(n.lib.brook_skeletonize(ctx, ctypes.byref(vol), ctypes.byref(opts), ctypes.byref(host)))
    dv = n.SkeletonsDeviceView()
    assert n.lib.brook_skeletons_get_device_view(host, ctypes.byref(dv)) == n.INVALID_ARGUMENT
    expected = n.packed_arrays(host)
    opts.flags |= n.DEVICE_OUTPUT
    dev = ctypes.c_void_p()
    n.check(n.lib.brook_skeletonize(ctx, ctypes.byref(vol), ctypes.byref(opts), ctypes.byref(dev)))
    n.check(n.lib.brook_skeletons_get_device_view(dev, ctypes.byref(dv)))
    nv, ne = dv.vertex_count, dv.edge_count
    assert dv.skeleton_count == len(expected["labels"]) and nv == len(expected["radii"]) and ne == len(expected["edges"])
    assert dv.vertices.memory == 1 and tuple(dv.vertices.shape) == (3, nv, 1) and tuple(dv.edges.shape) == (2, ne, 1)
    got = {}
    for name, which, dtype, shape in (("vertices", n.VERTICES, np.float32, (nv, 3)), ("edges", n.EDGES, np.uint32, (ne, 2)),
                                      ("radii", n.RADII, np.float32, (nv,))):
        arr = ctypes.c_void_p()
        n.check(n.lib.brook_skeletons_get_array(dev, which, ctypes.byref(arr)))
        buf = np.zeros(shape, dtype)
        n.check(n.lib.brook_array_copy_to_host(arr, buf.ctypes.data, buf.nbytes))
        n.lib.brook_array_destroy(arr)  # the array handle shares the result's storage
        got[name] = buf
    for name in ("vertices", "edges", "radii"):
        np.testing.assert_array_equal(got[name], expected[name], err_msg=name)
    copied = n.packed_arrays(dev)  # get_view on a device result, then destroy
    for name in ("labels", "v_off", "e_off", "vertices", "edges", "radii"):
        np.testing.assert_array_equal(copied[name], expected[name], err_msg=name)


def test_pinned_host_input_by_slabs_matches_device_input(gpu):
    """Host input in page-locked memory (256 MiB of uint64 here) is copied in slabs on a copy stream
    and the components' unions start on each slab as it arrives: the same skeletons as device
    input, also with object_ids (which waits for every slab first)."""
    import torch
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((512, 256, 256), objects=12, seed=21).astype(np.uint64)
    dev = torch.from_numpy(np.ascontiguousarray(labels.transpose(2, 1, 0))).cuda().permute(2, 1, 0)
    pinned_t = torch.empty(labels.shape[::-1], dtype=torch.uint64, pin_memory=True)
    pinned_t.numpy()[...] = labels.transpose(2, 1, 0)
    pinned = pinned_t.numpy().transpose(2, 1, 0)
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100)
    chosen = [int(x) for x in np.unique(labels)[1:6:2]]
    for extra in ({}, {"object_ids": chosen}):
        a = bk().skeletonize(dev, output="packed", **opts, **extra)
        b = bk().skeletonize(pinned, output="packed", **opts, **extra)
        assert len(a) > 0
        np.testing.assert_array_equal(a.labels, b.labels)
        np.testing.assert_array_equal(a.v_off, b.v_off)
        np.testing.assert_array_equal(a.vertices, b.vertices)
        np.testing.assert_array_equal(a.edges, b.edges)
        np.testing.assert_array_equal(a.radii.view(np.uint32), b.radii.view(np.uint32))


def test_extra_targets_match_oracle(gpu):
    """extra_targets_before (traced first, after the border targets) and extra_targets_after
    (traced once no voxel is left), points on the background dropped (lockstep.cu:127-134,
    trace.cu:209-212)."""
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((64, 64, 64), objects=6, seed=3)
    pts = {l: np.argwhere(labels == l) for l in (1, 2, 3)}
    before = [tuple(pts[1][len(pts[1]) // 2]), tuple(pts[2][-1]), tuple(np.argwhere(labels == 0)[0])]
    after = [tuple(pts[3][0]), tuple(pts[1][-1]), tuple(int(c) - 64 for c in pts[2][len(pts[2]) // 2])]
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100)
    got = bk().skeletonize(labels, output="packed", extra_targets_before=before, extra_targets_after=after, **opts)
    exp = oracle.skeletonize(labels, threads=8, extra_targets_before=before, extra_targets_after=after, **opts)
    assert_same(got, exp, "extra targets")
    plain = oracle.skeletonize(labels, threads=8, **opts)
    assert not np.array_equal(exp.array("vertices"), plain.array("vertices"))  # the targets changed something
    with pytest.raises(Exception, match="outside"):
        bk().skeletonize(labels, output="packed", extra_targets_before=[(64, 0, 0)], **opts)


def test_packed_device_output_matches_host(gpu):
    """output="packed_device": torch CUDA tensors over the result's own device arrays (no copy),
    equal to the host route, and still valid after the call's other objects are gone."""
    import torch

    from brook_b200 import synthetic

    labels = synthetic.tube_volume((64, 64, 64), objects=8, seed=6)
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100)
    host = bk().skeletonize(labels, output="packed", **opts)
    dev = bk().skeletonize(labels, output="packed_device", **opts)
    assert isinstance(dev.vertices, torch.Tensor) and dev.vertices.is_cuda
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dev.labels, host.labels)
    np.testing.assert_array_equal(dev.v_off, host.v_off)
    np.testing.assert_array_equal(dev.vertices.cpu().numpy(), host.vertices)
    np.testing.assert_array_equal(dev.edges.cpu().numpy(), host.edges)
    np.testing.assert_array_equal(dev.radii.cpu().numpy(), host.radii)


def test_edt_matches_oracle(gpu):
    """The EDT alone, through the C ABI, on multi-label volumes with and without black border."""
    from brook_b200 import _native as n
    from brook_b200 import synthetic

    labels = synthetic.dense_volume((96, 80, 70), seeds=20, seed=9).astype(np.uint64)
    ctx = n.context(0)
    for aniso, bb in (((1, 1, 1), 0), ((8, 8, 40), 1), ((7.91, 7.91, 7.91), 0)):
        host = np.asfortranarray(labels)  # kept alive: the volume descriptor borrows its memory
        vol = n.host_volume(host)
        arr = ctypes.c_void_p()
        n.check(n.lib.brook_edt(ctx, ctypes.byref(vol), (ctypes.c_float * 3)(*aniso), bb, ctypes.byref(arr)))
        d = np.zeros(labels.shape, np.float32, order="F")
        n.check(n.lib.brook_array_copy_to_host(arr, d.ctypes.data, d.nbytes))
        n.lib.brook_array_destroy(arr)
        # the oracle's EDT takes component ids; ids of equal original labels coincide with the labels
        _, inv = np.unique(labels, return_inverse=True)
        ids = inv.reshape(labels.shape).astype(np.uint32)
        exp = oracle.edt(ids, aniso, bool(bb))
        np.testing.assert_array_equal(d.view(np.uint32), exp.view(np.uint32), err_msg=str(aniso))
