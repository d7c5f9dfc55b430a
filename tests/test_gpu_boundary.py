"""The drop-in boundary on the GPU: producer-stream fencing of device input, the C ABI's array
upload, DLPack exports and component labels, per-sample extra targets and device output of a
batch, and a loop bound that runs out on the device (the call fails, the next one succeeds)."""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from test_gpu_parity import CFG0_PARAMS, assert_same, bk

pytestmark = pytest.mark.gpu

OPTS = dict(teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100)


class DLDevice(ctypes.Structure):
    _fields_ = [("device_type", ctypes.c_int), ("device_id", ctypes.c_int32)]


class DLDataType(ctypes.Structure):
    _fields_ = [("code", ctypes.c_uint8), ("bits", ctypes.c_uint8), ("lanes", ctypes.c_uint16)]


class DLTensor(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("device", DLDevice), ("ndim", ctypes.c_int32), ("dtype", DLDataType),
                ("shape", ctypes.POINTER(ctypes.c_int64)), ("strides", ctypes.POINTER(ctypes.c_int64)),
                ("byte_offset", ctypes.c_uint64)]


class DLManagedTensor(ctypes.Structure):
    pass


DLManagedTensor._fields_ = [("dl_tensor", DLTensor), ("manager_ctx", ctypes.c_void_p),
                            ("deleter", ctypes.CFUNCTYPE(None, ctypes.POINTER(DLManagedTensor)))]


class DLPackVersion(ctypes.Structure):
    _fields_ = [("major", ctypes.c_uint32), ("minor", ctypes.c_uint32)]


class DLManagedTensorVersioned(ctypes.Structure):
    pass


DLManagedTensorVersioned._fields_ = [("version", DLPackVersion), ("manager_ctx", ctypes.c_void_p),
                                     ("deleter", ctypes.CFUNCTYPE(None, ctypes.POINTER(DLManagedTensorVersioned))),
                                     ("flags", ctypes.c_uint64), ("dl_tensor", DLTensor)]


def _late_labels(labels, stream):
    """`labels` as a Fortran-ordered CUDA tensor whose contents a kernel on `stream` writes only
    after a long spin, queued without waiting: the values are not there until that stream gets
    there."""
    import torch

    src = torch.from_numpy(np.ascontiguousarray(labels.transpose(2, 1, 0))).cuda()
    dst = torch.zeros_like(src)
    torch.cuda.synchronize()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        torch.cuda._sleep(200_000_000)  # ~0.1 s of device time before the copy
        dst.copy_(src)
    return dst.permute(2, 1, 0)


def test_device_input_waits_for_its_producer_stream(gpu):
    """A tensor still being written on a side stream: the call waits for that stream, given as
    `stream=` or as torch's current stream, and never reads the unwritten volume."""
    import torch

    from brook_b200 import synthetic

    labels = synthetic.tube_volume((64, 64, 64), objects=6, seed=4)
    expected = bk().skeletonize(labels, output="packed", **OPTS)
    assert len(expected) == 6
    side = torch.cuda.Stream()
    got = bk().skeletonize(_late_labels(labels, side), output="packed", stream=side, **OPTS)
    assert_same(got, oracle.skeletonize(labels, threads=8, **OPTS), "stream=")
    late = _late_labels(labels, side)
    with torch.cuda.stream(side):
        got = bk().skeletonize(late, output="packed", **OPTS)
    np.testing.assert_array_equal(got.vertices, expected.vertices)
    late = _late_labels(labels, side)
    batch = bk().skeletonize_batch([late], output="packed", stream=side.cuda_stream, **OPTS)
    np.testing.assert_array_equal(batch[0].vertices, expected.vertices)
    torch.cuda.synchronize()


def test_batch_per_sample_targets_match_oracle(gpu):
    """extra_targets_before / _after per sample of a batch (src/brook/batch.py:173-220): each
    sample's result equals the oracle on that sample with its own targets."""
    from brook_b200 import synthetic

    samples = [synthetic.tube_volume(shape, objects=5, seed=s)
               for s, shape in enumerate([(64, 48, 40), (40, 56, 64), (48, 48, 48)])]
    before, after = [], []
    for i, v in enumerate(samples):
        one, two = np.argwhere(v == 1), np.argwhere(v == 2)
        before.append([tuple(one[len(one) // 2])] if i != 1 else [])
        after.append([tuple(two[0]), tuple(one[-1])] if i != 0 else None)
    batch = bk().skeletonize_batch(samples, output="packed", extra_targets_before=before, extra_targets_after=after,
                                   **OPTS)
    changed = False
    for i, v in enumerate(samples):
        exp = oracle.skeletonize(v, threads=8, extra_targets_before=before[i], extra_targets_after=after[i] or (),
                                 **OPTS)
        assert_same(batch[i], exp, f"sample {i}")
        plain = oracle.skeletonize(v, threads=8, **OPTS)
        changed |= not np.array_equal(exp.array("vertices"), plain.array("vertices"))
    assert changed
    with pytest.raises(ValueError, match="per sample"):
        bk().skeletonize_batch(samples, output="packed", extra_targets_before=[(1, 2, 3)], **OPTS)
    with pytest.raises(ValueError, match="entries"):
        bk().skeletonize_batch(samples, output="packed", extra_targets_before=[[], []], **OPTS)


def test_batch_device_output_stays_on_device(gpu):
    """skeletonize_batch(output="packed_device") hands back the library's device arrays (torch CUDA
    tensors), equal to the host output."""
    import torch

    from brook_b200 import synthetic

    samples = [synthetic.tube_volume((48, 40, 56), objects=4, seed=s) for s in range(3)]
    host = bk().skeletonize_batch(samples, output="packed", **OPTS)
    dev = bk().skeletonize_batch(samples, output="packed_device", **OPTS)
    assert dev.on_device and dev.vertices.is_cuda and dev.edges.dtype == torch.uint32
    np.testing.assert_array_equal(dev.s_off, host.s_off)
    np.testing.assert_array_equal(dev.labels, host.labels)
    np.testing.assert_array_equal(dev.vertices.cpu().numpy(), host.vertices)
    np.testing.assert_array_equal(dev.edges.view(torch.int32).cpu().numpy().view(np.uint32), host.edges)
    np.testing.assert_array_equal(dev.radii.cpu().numpy(), host.radii)
    for i in range(3):
        np.testing.assert_array_equal(dev[i].vertices, host[i].vertices)


def test_loop_bound_fails_the_call_and_the_next_call_succeeds(gpu, monkeypatch):
    """The engine's round bounds are the guard against a flood that does not end: a test cap of
    two rounds makes them run out on the device; the call returns an error (no hang, no fault)
    and the same context then skeletonizes correctly."""
    from brook_b200 import _native, synthetic

    labels = synthetic.tube_volume((48, 48, 48), objects=4, seed=2)
    monkeypatch.setenv("BROOK_B200_TEST_ROUND_LIMIT", "2")
    with pytest.raises(_native.BrookError, match="loop bound") as failure:
        bk().skeletonize(labels, output="packed", **OPTS)
    assert failure.value.status == _native.INTERNAL_ERROR
    monkeypatch.delenv("BROOK_B200_TEST_ROUND_LIMIT")
    got = bk().skeletonize(labels, output="packed", **OPTS)
    assert len(got) == 4
    assert_same(got, oracle.skeletonize(labels, threads=8, **OPTS), "after a failed call")


def _capsule(ptr, name):
    make = ctypes.pythonapi.PyCapsule_New
    make.restype = ctypes.py_object
    make.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
    return make(ptr, name, None)


def test_c_abi_upload_dlpack_and_component_labels(gpu):
    """brook_array_upload (host C order, host strided, device input; float and integer types),
    brook_array_to_dlpack(_versioned) consumed by torch and by hand, brook_components_labels."""
    import torch

    from brook_b200 import _native as n
    from brook_b200 import synthetic

    lib, ctx = n.lib, n.context(0)
    rng = np.random.default_rng(3)
    for host in (rng.integers(0, 1 << 40, (20, 17, 9), dtype=np.uint64),
                 np.ascontiguousarray(rng.random((13, 11, 7), dtype=np.float32)),
                 rng.integers(-5, 5, (30, 20, 10), dtype=np.int16)[::2, 1::2, ::-1]):
        vol = n.host_volume(host)
        arr = ctypes.c_void_p()
        n.check(lib.brook_array_upload(ctx, ctypes.byref(vol), ctypes.byref(arr)))
        out = np.zeros(host.shape, host.dtype, order="F")
        n.check(lib.brook_array_copy_to_host(arr, out.ctypes.data, out.nbytes))
        np.testing.assert_array_equal(out, host)
        view = n.Volume()
        n.check(lib.brook_array_view(arr, ctypes.byref(view)))
        assert tuple(view.shape) == host.shape and view.memory == n.DEVICE
        # zero-copy into torch; the export outlives the array handle
        dl = ctypes.c_void_p()
        n.check(lib.brook_array_to_dlpack(arr, ctypes.byref(dl)))
        lib.brook_array_destroy(arr)
        t = torch.utils.dlpack.from_dlpack(_capsule(dl.value, b"dltensor"))
        assert t.is_cuda and tuple(t.shape) == host.shape
        np.testing.assert_array_equal(t.cpu().numpy(), host)
        del t
    # a device C-ordered source, and the versioned export read by hand
    src = torch.arange(4 * 5 * 6, dtype=torch.int32, device="cuda").reshape(4, 5, 6)
    vol = n.device_volume(src.data_ptr(), tuple(src.shape), [s * 4 for s in src.stride()], np.int32)
    arr = ctypes.c_void_p()
    torch.cuda.synchronize()
    n.check(lib.brook_array_upload(ctx, ctypes.byref(vol), ctypes.byref(arr)))
    dlv = ctypes.c_void_p()
    n.check(lib.brook_array_to_dlpack_versioned(arr, 7, ctypes.byref(dlv)))
    m = ctypes.cast(dlv, ctypes.POINTER(DLManagedTensorVersioned)).contents
    assert (m.version.major, m.version.minor) == (1, 1) and m.flags == 0
    t = m.dl_tensor
    assert t.device.device_type == 2 and t.ndim == 3 and (t.dtype.code, t.dtype.bits) == (0, 32)
    assert [t.shape[i] for i in range(3)] == [4, 5, 6] and [t.strides[i] for i in range(3)] == [1, 4, 20]
    got = np.zeros(120, np.int32)
    n.check(lib.brook_array_copy_to_host(arr, got.ctypes.data, got.nbytes))
    np.testing.assert_array_equal(got.reshape(6, 5, 4).transpose(2, 1, 0), src.cpu().numpy())
    m.deleter(ctypes.cast(dlv, ctypes.POINTER(DLManagedTensorVersioned)))
    lib.brook_array_destroy(arr)
    # component ids as an array handle that outlives the components handle
    labels = np.asfortranarray(synthetic.tube_volume((40, 36, 30), objects=5, seed=1))
    vol = n.host_volume(labels)
    cc = ctypes.c_void_p()
    n.check(lib.brook_connected_components(ctx, ctypes.byref(vol), ctypes.byref(cc)))
    cview = n.Volume()
    count = ctypes.c_size_t()
    n.check(lib.brook_components_view(cc, ctypes.byref(cview), None, None, ctypes.byref(count)))
    ids = np.zeros(labels.shape, n.DTYPE_NAMES[cview.dtype], order="F")
    n.check(lib.brook_components_copy_to_host(cc, ids.ctypes.data, ids.nbytes))
    arr = ctypes.c_void_p()
    n.check(lib.brook_components_labels(cc, ctypes.byref(arr)))
    lib.brook_components_destroy(cc)
    again = np.zeros_like(ids)
    n.check(lib.brook_array_copy_to_host(arr, again.ctypes.data, again.nbytes))
    lib.brook_array_destroy(arr)
    np.testing.assert_array_equal(again, ids)
    assert count.value > 0 and ids.max() == count.value
