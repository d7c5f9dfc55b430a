"""Post-processing of PackedSkeletons on the GPU: the reference's brook.device_post
(src/brook/_device_post.py:1-49) over this library's C ABI (brook_postprocess_canonical,
brook_postprocess_step, brook_skeleton_components).

Each function takes PackedSkeletons on the host or the device and returns new PackedSkeletons on
the device (`.to_host()` copies them back); every label of the input stays, possibly empty.
"""
from __future__ import annotations

import ctypes

from . import _native
from ._packed import PackedSkeletons

REMOVE_DUST, REMOVE_LOOPS, JOIN_COMPONENTS, REMOVE_TICKS, PRUNE_UNUSED = 1, 2, 3, 4, 5


def _call(p, fn, *args, device=0):
    lib = _native.load()
    ctx = _native.context(device)
    handle = _native.skeletons_handle(p, device)
    out = ctypes.c_void_p()
    try:
        _native.check(getattr(lib, fn)(ctx, handle, *args, ctypes.byref(out)))
    finally:
        lib.brook_skeletons_destroy(handle)
    return PackedSkeletons.from_arrays(_native.packed_device_arrays(out))


def components(p, device=0):
    """A connected-component id for every packed vertex (the smallest global vertex index of its
    component; int64, on the GPU)."""
    lib = _native.load()
    handle = _native.skeletons_handle(p, device)
    arr = ctypes.c_void_p()
    try:
        _native.check(lib.brook_skeleton_components(_native.context(device), handle, ctypes.byref(arr)))
    finally:
        lib.brook_skeletons_destroy(handle)
    return _native.array_tensor(arr)


def remove_dust(p, dust_threshold, device=0):
    """Removes connected components whose cable length is below `dust_threshold` (physical units)."""
    if dust_threshold == 0 or int(p.v_off[-1]) == 0:
        return p
    return _call(p, "brook_postprocess_step", REMOVE_DUST, float(dust_threshold), device=device)


def remove_loops(p, device=0):
    """Breaks the cycles of each skeleton."""
    return _call(p, "brook_postprocess_step", REMOVE_LOOPS, 0.0, device=device)


def join_close_components(p, device=0):
    """Joins the connected components of each skeleton into one tree where they come within twice
    the skeleton's largest radius."""
    return _call(p, "brook_postprocess_step", JOIN_COMPONENTS, 0.0, device=device)


def remove_ticks(p, tick_threshold, device=0):
    """Removes terminal branches shorter than `tick_threshold` (physical units)."""
    return _call(p, "brook_postprocess_step", REMOVE_TICKS, float(tick_threshold), device=device)


def prune_unused(p, device=0):
    """Drops the vertices on no edge."""
    return _call(p, "brook_postprocess_step", PRUNE_UNUSED, 0.0, device=device)


def postprocess(p, dust_threshold=1500, tick_threshold=3500, device=0):
    """Dust, loops, joins and ticks with the reference's tie rules, then the vertices on no edge
    are dropped. Returns new PackedSkeletons on the device."""
    return _call(p, "brook_postprocess_canonical", float(dust_threshold), float(tick_threshold), device=device)


__all__ = ["components", "remove_dust", "remove_loops", "join_close_components", "remove_ticks", "prune_unused",
           "postprocess"]
