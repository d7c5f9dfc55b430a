"""brook_edt_device_noalloc: the EDT for callers that cannot allocate device memory (for example
code running inside another framework's memory budget, where the free device memory belongs to
that framework's caching allocator). It must give brook_edt's result, call after call, while
using only its fixed scratch; its inputs and outputs here are the test's own torch tensors.

This file is collected last so that a failure here cannot hide the results of the other tests."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _edt_reference(labels, aniso, black_border):
    """brook_edt (the allocating entry point) on host labels."""
    from brook_b200 import _native as n

    arr = ctypes.c_void_p()
    host = np.asfortranarray(labels)  # kept alive: the volume descriptor borrows its memory
    vol = n.host_volume(host)
    n.check(n.lib.brook_edt(n.context(0), ctypes.byref(vol), (ctypes.c_float * 3)(*aniso), int(black_border),
                            ctypes.byref(arr)))
    out = np.zeros(labels.shape, np.float32, order="F")
    n.check(n.lib.brook_array_copy_to_host(arr, out.ctypes.data, out.nbytes))
    n.lib.brook_array_destroy(arr)
    return out


def _edt_noalloc(labels_dev, out_dev, aniso, black_border, stream):
    from brook_b200 import _native as n

    vol = n.device_volume(labels_dev.data_ptr(), tuple(labels_dev.shape),
                          [s * 4 for s in labels_dev.stride()], np.uint32)
    return n.lib.brook_edt_device_noalloc(ctypes.byref(vol), (ctypes.c_float * 3)(*aniso), int(black_border),
                                          ctypes.c_void_p(out_dev.data_ptr()), ctypes.c_void_p(stream.cuda_stream))


def _device_fortran(labels):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(labels.transpose(2, 1, 0))).cuda()
    return t.permute(2, 1, 0)  # (x, y, z) view, x fastest


def test_noalloc_edt_matches_brook_edt_twice(gpu):
    import torch

    from brook_b200 import _native as n
    from brook_b200 import synthetic

    first = synthetic.tube_volume((70, 60, 50), objects=6, seed=41)
    second = synthetic.dense_volume((96, 80, 64), seeds=15, seed=42)
    _, inv = np.unique(second, return_inverse=True)
    second = inv.reshape(second.shape).astype(np.uint32)
    stream = torch.cuda.Stream()
    # two calls in a row on the same stream, different volumes, spacings and borders
    cases = [(first, (16.0, 16.0, 40.0), False), (second, (7.91, 7.91, 7.91), True)]
    outs = []
    with torch.cuda.stream(stream):
        for labels, aniso, bb in cases:
            dev = _device_fortran(labels.astype(np.uint32))
            out = torch.empty(labels.size, dtype=torch.float32, device="cuda")
            status = _edt_noalloc(dev, out, aniso, bb, stream)
            assert status == n.SUCCESS, n.lib.brook_last_error().decode()
            outs.append((dev, out))
    stream.synchronize()
    for (labels, aniso, bb), (_, out) in zip(cases, outs):
        got = out.cpu().numpy().reshape(labels.shape[::-1]).transpose(2, 1, 0)
        exp = _edt_reference(labels.astype(np.uint32), aniso, bb)
        np.testing.assert_array_equal(got.view(np.uint32), exp.view(np.uint32), err_msg=str(aniso))


def test_noalloc_edt_over_several_stack_batches(gpu):
    """A volume whose y and z passes need more envelope stack than the fixed scratch holds at
    once (256 x 256 x 64: about 68 MB of y-pass stacks), so each pass runs in several batches of
    lines over the same scratch; twice in a row, equal to brook_edt bit for bit."""
    import torch

    from brook_b200 import _native as n
    from brook_b200 import synthetic

    labels = synthetic.dense_volume((256, 256, 64), seeds=25, seed=43)
    _, inv = np.unique(labels, return_inverse=True)
    labels = inv.reshape(labels.shape).astype(np.uint32)
    exp = _edt_reference(labels, (8.0, 8.0, 40.0), False)
    dev = _device_fortran(labels)
    stream = torch.cuda.Stream()
    for _ in range(2):
        out = torch.full((labels.size,), -1.0, dtype=torch.float32, device="cuda")
        with torch.cuda.stream(stream):
            status = _edt_noalloc(dev, out, (8.0, 8.0, 40.0), False, stream)
        assert status == n.SUCCESS, n.lib.brook_last_error().decode()
        stream.synchronize()
        got = out.cpu().numpy().reshape(labels.shape[::-1]).transpose(2, 1, 0)
        np.testing.assert_array_equal(got.view(np.uint32), exp.view(np.uint32))


def test_noalloc_edt_rejects_what_does_not_fit(gpu):
    import torch

    from brook_b200 import _native as n

    wide = torch.ones((13000, 1, 1), dtype=torch.int32, device="cuda").to(torch.uint32)
    out = torch.empty(13000, dtype=torch.float32, device="cuda")
    status = _edt_noalloc(wide, out, (1.0, 1.0, 1.0), False, torch.cuda.current_stream())
    assert status == n.INVALID_ARGUMENT
    assert "fixed 32 MiB scratch" in n.lib.brook_last_error().decode()
