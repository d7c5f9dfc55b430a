"""`skeletonize`: the reference's brook.skeletonize argument surface (src/brook/_intake.py:99-103)
over the brook_b200 C ABI."""
from __future__ import annotations

import os
import warnings

import numpy as np

from . import _native
from ._packed import PackedSkeletons

# The values of the reference's brook.DEFAULT_TEASAR_PARAMS (src/brook/__init__.py:8-17).
DEFAULT_TEASAR_PARAMS = {
    "scale": 1.5,
    "const": 300,
    "pdrf_scale": 100000,
    "pdrf_exponent": 4,
    "soma_acceptance_threshold": 3500,
    "soma_detection_threshold": 750,
    "soma_invalidation_const": 300,
    "soma_invalidation_scale": 2,
}

# Keys a caller leaves out take kimimaro.trace's defaults, as in the reference (skeleton.hpp:23-27).
TRACE_DEFAULTS = {
    "scale": 10.0, "const": 10.0, "pdrf_scale": 5000.0, "pdrf_exponent": 16.0,
    "soma_detection_threshold": 1100.0, "soma_acceptance_threshold": 4000.0,
    "soma_invalidation_scale": 0.5, "soma_invalidation_const": 0.0, "max_paths": None,
}


# Device bytes per voxel of an in-core call beyond its labels (the largest measured peak is 157 B at
# 512^3), and the share of the free device memory an in-core call may take before skeletonize
# streams the volume instead (the reference's rule, src/brook/_intake.py:43-56).
_INCORE_BYTES_PER_VOXEL = 160
_INCORE_MEMORY_FRACTION = 0.5


class DimensionError(Exception):
    """The input volume has unsupported dimensions."""


def teasar(params):
    out = dict(TRACE_DEFAULTS)
    for key, value in dict(params).items():
        if key not in out:
            raise TypeError(f"unexpected TEASAR parameter: {key}")
        out[key] = value if key == "max_paths" else float(value)
    return out


def format_labels(labels):
    """Host labels as a 3D integer NumPy array (bool -> uint8, trailing singleton axes dropped,
    missing axes appended), without rearranging its bytes."""
    labels = np.asarray(labels)
    if labels.dtype == bool:
        labels = labels.view(np.uint8)
    while labels.ndim > 3 and labels.shape[-1] == 1:
        labels = labels[..., 0]
    if labels.ndim > 3:
        raise DimensionError(f"{labels.ndim} dimensions is not supported (max 3).")
    while labels.ndim < 3:
        labels = labels[..., np.newaxis]
    if labels.dtype.kind not in "ui":
        raise TypeError("brook_b200: labels must be integer or boolean")
    return labels


def _is_device(labels):
    return not isinstance(labels, np.ndarray) and (hasattr(labels, "__cuda_array_interface__") or
                                                   (hasattr(labels, "is_cuda") and labels.is_cuda))


def producer_stream(labels, stream=None):
    """The stream handle whose queued work must finish before `labels` (device memory) is read:
    the caller's `stream` (an int handle or a torch.cuda.Stream), else torch's current stream for a
    torch tensor, else the array's own CUDA array interface stream, else the legacy default
    stream. Handles follow the CUDA array interface: 1 legacy default, 2 per-thread default,
    anything else a cudaStream_t. (The reference's binding fences the same producer,
    cpp/python/bindings.cpp:104-126.)"""
    if stream is not None:
        handle = getattr(stream, "cuda_stream", stream)
        return int(handle) or 1
    try:
        import torch
    except ImportError:  # pragma: no cover
        torch = None
    if torch is not None and isinstance(labels, torch.Tensor):
        return int(torch.cuda.current_stream(labels.device).cuda_stream) or 1
    cai = getattr(labels, "__cuda_array_interface__", None)
    if cai is not None and cai.get("stream") is not None:
        return int(cai["stream"]) or 1
    return 1


def device_volume(labels):
    """(brook_volume, keep-alive) for a CUDA array (torch tensor or an object with the CUDA array
    interface); the array is read in place when it is Fortran-ordered."""
    try:
        import torch
    except ImportError:  # pragma: no cover
        torch = None
    if torch is not None and isinstance(labels, torch.Tensor):
        t = labels
        if t.dtype == torch.bool:
            t = t.view(torch.uint8)
        while t.dim() < 3:
            t = t.unsqueeze(-1)
        dtype = np.dtype(str(t.dtype).replace("torch.", ""))
        strides = [s * t.element_size() for s in t.stride()]
        return _native.device_volume(t.data_ptr(), tuple(t.shape), strides, dtype), t
    cai = labels.__cuda_array_interface__
    shape = tuple(cai["shape"])
    dtype = np.dtype(cai["typestr"])
    strides = cai.get("strides") or tuple(int(np.prod(shape[a + 1:])) * dtype.itemsize for a in range(len(shape)))
    while len(shape) < 3:
        shape, strides = shape + (1,), tuple(strides) + (dtype.itemsize,)
    return _native.device_volume(cai["data"][0], shape, strides, dtype), labels


def _use_streaming(streaming, labels, device):
    """streaming as given; else BROOK_STREAMING (0 / off / false / no: in-core); else stream when the
    in-core state would take more than half the device's free memory, or the volume holds 2^31
    voxels or more (in-core calls index voxels with 31 bits)."""
    if streaming is not None:
        return bool(streaming)
    env = os.environ.get("BROOK_STREAMING", "").strip().lower()
    if env:
        return env not in ("0", "off", "false", "no")
    if labels.size >= (1 << 31) - 1:
        return True
    need = int(labels.size) * (labels.dtype.itemsize + _INCORE_BYTES_PER_VOXEL)
    if need < (1 << 30):
        return False
    import torch

    free, _ = torch.cuda.mem_get_info(device)
    return need > _INCORE_MEMORY_FRACTION * free


def _run_streamed(volume, params, anisotropy, object_ids, dust_threshold, fix_branching, fix_borders, extra_before,
                  extra_after, device, device_output=False, budget=0):
    """brook_skeletonize_streamed over a host volume, as PackedSkeletons."""
    ctypes = _native.ctypes
    opts = _native.options(params, anisotropy, dust_threshold, fix_branching, fix_borders, object_ids,
                           extra_before, extra_after)
    if device_output:
        opts.flags |= _native.DEVICE_OUTPUT
    lib = _native.load()
    out = ctypes.c_void_p()
    _native.check(lib.brook_skeletonize_streamed(_native.context(device), ctypes.byref(volume), ctypes.byref(opts),
                                                 int(budget), ctypes.byref(out)))
    grab = _native.packed_device_arrays if device_output else _native.packed_arrays
    return PackedSkeletons.from_arrays(grab(out.value))


def _run(volumes, params, anisotropy, object_ids, dust_threshold, fix_branching, fix_borders, extra_before,
         extra_after, device, device_output=False, producers=(), sample_targets=None, fill_holes=False,
         fix_avocados=False):
    """One C call over `volumes`, as PackedSkeletons. producers: stream handles the library's
    stream waits for first (the producers of device inputs). sample_targets: per volume (before,
    after) point lists of a batch (extra_before / extra_after then stay empty)."""
    handles = _run_handles(volumes, params, anisotropy, object_ids, dust_threshold, fix_branching, fix_borders,
                           extra_before, extra_after, device, device_output, producers, sample_targets, fill_holes,
                           fix_avocados)
    grab = _native.packed_device_arrays if device_output else _native.packed_arrays
    return [PackedSkeletons.from_arrays(grab(h)) for h in handles]


def _run_handles(volumes, params, anisotropy, object_ids, dust_threshold, fix_branching, fix_borders, extra_before,
                 extra_after, device, device_output=False, producers=(), sample_targets=None, fill_holes=False,
                 fix_avocados=False):
    """_run's C call; returns the raw result handles (the caller destroys them)."""
    ctypes = _native.ctypes
    opts = _native.options(params, anisotropy, dust_threshold, fix_branching, fix_borders, object_ids,
                           extra_before, extra_after)
    if device_output:
        opts.flags |= _native.DEVICE_OUTPUT
    if fill_holes:
        opts.flags |= _native.FILL_HOLES
    if fix_avocados:
        opts.flags |= _native.FIX_AVOCADOS
    lib = _native.load()
    ctx = _native.context(device)
    for handle in dict.fromkeys(producers):
        _native.check(lib.brook_context_wait_stream(ctx, int(handle)))
    count = len(volumes)
    arr = (_native.Volume * max(count, 1))(*volumes)
    handles = (ctypes.c_void_p * max(count, 1))()
    if sample_targets is not None:
        table = (_native.SampleTargets * max(count, 1))()
        keep = []
        for i, (before, after) in enumerate(sample_targets):
            for name, points in (("before", before), ("after", after)):
                pts = np.ascontiguousarray(np.asarray(list(points), np.int64).reshape(-1, 3))
                keep.append(pts)
                if pts.size:
                    setattr(table[i], name, pts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
                    setattr(table[i], name + "_count", pts.shape[0])
        _native.check(lib.brook_skeletonize_batch_targets(ctx, arr, count, ctypes.byref(opts), table, handles))
    elif count == 1:
        _native.check(lib.brook_skeletonize(ctx, arr, ctypes.byref(opts), handles))
    else:
        _native.check(lib.brook_skeletonize_batch(ctx, arr, count, ctypes.byref(opts), handles))
    return [handles[i] for i in range(count)]


def skeletonize(all_labels, teasar_params=DEFAULT_TEASAR_PARAMS, anisotropy=(1, 1, 1), object_ids=None,
                dust_threshold=1000, progress=False, fix_branching=True, in_place=False, fix_borders=True, parallel=1,
                parallel_chunk_size=100, extra_targets_before=(), extra_targets_after=(), fill_holes=False,
                fix_avocados=False, voxel_graph=None, streaming=None, output="skeletons", stream=None, borrow=True,
                device=0):
    """Skeletonize a 3D label volume on a B200; a drop-in for the reference's `brook.skeletonize`
    (and so for `kimimaro.skeletonize`).

    Returns `{label: Skeleton}` for output="skeletons", `PackedSkeletons` (host arrays) for
    "packed", and the same with CUDA tensors for "packed_device". Device input: a torch CUDA
    tensor or an array with the CUDA array interface, read in place when Fortran-ordered; the
    library's stream first waits for the producer's work (`stream`: the producer's stream handle
    or torch.cuda.Stream; default: the array's own CUDA array interface stream, torch's current
    stream for a torch tensor, else the legacy default stream). `fill_holes` fills every
    component's voids before the distance transform (the reference's rule: components in
    ascending id, a component whose voxels an earlier fill painted is not filled);
    `fix_avocados` merges pits (an object whose distance field passes soma_detection_threshold / 2.5
    and that another object encloses) into the objects around them (Kimimaro's rule). `parallel`,
    `streaming` (host input only): None streams when the in-core state would take more than half
    the device's free memory (BROOK_STREAMING overrides), True always, False never; a streamed call
    gives the same skeletons within a device budget (BROOK_STREAM_BUDGET_MB, default a quarter of
    the free memory) and refuses fill_holes / fix_avocados, as the reference's does.
    `parallel_chunk_size`, `in_place`, `progress` and `borrow` are accepted for compatibility.
    `voxel_graph` is not supported by this build and raises.
    """
    if output not in ("skeletons", "packed", "packed_device"):
        raise ValueError("brook_b200: output must be 'skeletons', 'packed' or 'packed_device'")
    if voxel_graph is not None:
        raise NotImplementedError("brook_b200: voxel_graph is not supported")
    params = teasar(teasar_params)
    anisotropy = tuple(float(a) for a in np.asarray(anisotropy, dtype=np.float32))
    producers = []
    streamed = False
    if _is_device(all_labels):
        if streaming:
            raise NotImplementedError("streaming is a host-input feature")
        volume, keep = device_volume(all_labels)
        producers.append(producer_stream(all_labels, stream))
    else:
        keep = format_labels(all_labels)
        if keep.size <= dust_threshold:
            packed = PackedSkeletons.empty(anisotropy)
            return {} if output == "skeletons" else packed
        streamed = _use_streaming(streaming, keep, device)
        if streamed and (fill_holes or fix_avocados):
            raise NotImplementedError("brook streaming mode does not support voxel_graph, fill_holes or fix_avocados; "
                                      "pass streaming=False or process the volume in chunks.")
        if streamed and streaming is None and not os.environ.get("BROOK_STREAMING", "").strip():
            warnings.warn(f"brook_b200: a {tuple(keep.shape)} volume does not fit in GPU memory; it is streamed "
                          "(components by slabs, each traced component in its bounding box). "
                          "brook_b200.skeletonize_chunked() processes overlapping chunks at in-core speed.",
                          stacklevel=2)
        volume = _native.host_volume(keep)
    ids = None if object_ids is None else [int(i) for i in object_ids]
    before = [tuple(int(c) for c in p) for p in extra_targets_before]
    after = [tuple(int(c) for c in p) for p in extra_targets_after]
    if streamed:
        packed = _run_streamed(volume, params, anisotropy, ids, dust_threshold, fix_branching, fix_borders, before,
                               after, device, device_output=output == "packed_device")
    else:
        packed = _run([volume], params, anisotropy, ids, dust_threshold, fix_branching, fix_borders, before, after,
                      device, device_output=output == "packed_device", producers=producers, fill_holes=fill_holes,
                      fix_avocados=fix_avocados)[0]
    del keep
    if output == "skeletons":
        return packed.to_skeletons()
    return packed
