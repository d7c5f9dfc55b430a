"""Volumes in overlapping chunks, and the merge of skeleton fragments: the reference's
skeletonize_chunked (src/brook/_pool.py:361-409, on one GPU here) and merge_fragments
(src/brook/_packed.py:98-111).

A volume larger than the device's memory is cut into chunks that overlap by `overlap` voxels
(iter_chunks); the chunks run through skeletonize_batch a few at a time (the device's
free-memory budget bounds each group), their results stay on the device, and one device merge
(brook_merge_skeletons) joins the fragments, each shifted to its chunk's physical origin.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from ._intake import DEFAULT_TEASAR_PARAMS, _run_handles, format_labels, teasar
from ._packed import PackedSkeletons
from .sharding import iter_chunks

# device bytes per voxel of one chunk in flight: the labels and the per-voxel state of a call
# (the serving loop's measured footprint)
_STATE_BYTES_PER_VOXEL = 160


def physical_origins(starts, anisotropy):
    """Chunk starts (voxels) as physical origins: float32(start * spacing) per axis, as the
    reference computes them (cpp/python/scheduling_bindings.cpp:59-63)."""
    a = np.asarray(anisotropy, np.float32)
    return [tuple(float(np.float32(np.float32(s[k]) * a[k])) for k in range(3)) for s in starts]


def _merge_handles(handles, origins, device):
    """The brook_merge_skeletons device result of fragment handles (the caller destroys it)."""
    lib = _native.load()
    ctx = _native.context(device)
    arr = (ctypes.c_void_p * max(len(handles), 1))(*handles)
    flat = (ctypes.c_float * max(3 * len(origins), 1))(*[c for o in origins for c in o])
    out = ctypes.c_void_p()
    _native.check(lib.brook_merge_skeletons(ctx, arr, flat, len(handles), ctypes.byref(out)))
    return out.value


def _postprocessed(handle, postprocess, device):
    """The canonical device post-processing of a result handle (which it destroys), as a new
    handle; `postprocess` is a dict of dust_threshold / tick_threshold (defaults 1500 / 3500)."""
    lib = _native.load()
    post = dict(postprocess)
    unknown = set(post) - {"dust_threshold", "tick_threshold"}
    if unknown:
        lib.brook_skeletons_destroy(handle)
        raise TypeError(f"brook_b200: unknown postprocess keys {sorted(unknown)}")
    out = ctypes.c_void_p()
    try:
        _native.check(lib.brook_postprocess_canonical(_native.context(device), handle,
                                                      float(post.get("dust_threshold", 1500)),
                                                      float(post.get("tick_threshold", 3500)), ctypes.byref(out)))
    finally:
        lib.brook_skeletons_destroy(handle)
    return out.value


def merge_fragments(parts, origins, on_device=False, device=0):
    """Merges PackedSkeletons fragments (host or device) placed at `origins` (physical units)
    into one skeleton per label, on the device; the result stays there when `on_device`."""
    parts, origins = list(parts), [tuple(float(c) for c in o) for o in origins]
    if len(parts) != len(origins):
        raise ValueError("fragment/origin count mismatch")
    lib = _native.load()
    handles = []
    try:
        for p in parts:
            handles.append(_native.skeletons_handle(p, device))
        merged = _merge_handles(handles, origins, device)
    finally:
        for h in handles:
            lib.brook_skeletons_destroy(h)
    grab = _native.packed_device_arrays if on_device else _native.packed_arrays
    return PackedSkeletons.from_arrays(grab(merged))


def skeletonize_chunked(all_labels, chunk_shape=(512, 512, 512), overlap=1, teasar_params=DEFAULT_TEASAR_PARAMS,
                        anisotropy=(1, 1, 1), dust_threshold=1000, fix_branching=True, output="skeletons",
                        postprocess=None, postprocess_engine="device", memory_budget=None, device=0):
    """Skeletonizes a host volume in chunks of `chunk_shape` overlapping by `overlap` voxels
    (border targets on, as the reference forces) and merges the fragments. Returns
    {label: Skeleton}, PackedSkeletons ("packed") or the same on the device ("packed_device").
    `postprocess` (a dict of dust_threshold / tick_threshold) runs the canonical post-processing
    on the merged skeletons on the GPU (postprocess_engine "device", the reference's default;
    its "kimimaro" CPU engine is not part of this library). `memory_budget` (bytes, default: 80 %
    of the device's free memory) bounds the chunks run together."""
    if postprocess_engine not in ("device", "kimimaro"):
        raise ValueError("brook_b200: postprocess_engine must be 'device' or 'kimimaro'")
    if postprocess is not None and postprocess_engine != "device":
        raise NotImplementedError("brook_b200: the CPU (kimimaro) post-processing engine is not part of this library")
    if output not in ("skeletons", "packed", "packed_device"):
        raise ValueError("brook_b200: output must be 'skeletons', 'packed' or 'packed_device'")
    labels = format_labels(all_labels)
    params = teasar(teasar_params)
    anisotropy = tuple(float(a) for a in np.asarray(anisotropy, dtype=np.float32))
    slices = list(iter_chunks(labels.shape, chunk_shape, overlap))
    if memory_budget is None:
        import torch

        free, _ = torch.cuda.mem_get_info(device)
        memory_budget = 0.8 * free
    lib = _native.load()
    handles, origins = [], []
    try:
        group, group_bytes = [], 0
        starts = [[sl.start for sl in chunk] for chunk in slices]

        def flush():
            nonlocal group, group_bytes
            if not group:
                return
            chunks = [np.asfortranarray(labels[slices[i]]) for i in group]
            volumes = [_native.host_volume(c) for c in chunks]
            handles.extend(_run_handles(volumes, params, anisotropy, None, dust_threshold, fix_branching, True, [], [],
                                        device, device_output=True))
            origins.extend(physical_origins([starts[i] for i in group], anisotropy))
            group, group_bytes = [], 0

        for i, chunk in enumerate(slices):
            n = int(np.prod([sl.stop - sl.start for sl in chunk]))
            need = n * (labels.dtype.itemsize + _STATE_BYTES_PER_VOXEL)
            if group and group_bytes + need > memory_budget:
                flush()
            group.append(i)
            group_bytes += need
        flush()
        merged = _merge_handles(handles, origins, device)
    finally:
        for h in handles:
            lib.brook_skeletons_destroy(h)
    if postprocess is not None:
        merged = _postprocessed(merged, postprocess, device)
    grab = _native.packed_device_arrays if output == "packed_device" else _native.packed_arrays
    merged = PackedSkeletons.from_arrays(grab(merged))
    if output == "skeletons":
        return merged.to_skeletons()
    return merged


__all__ = ["skeletonize_chunked", "merge_fragments", "physical_origins"]
