"""ctypes binding of the C ABI in include/brook_b200.h (libbrook_b200.so, built in-tree).

The library is the only compute path. It is loaded on first use (`load()`, or the module
attribute `lib`), so that importing the package costs nothing; a missing library fails loudly
there, with no fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libbrook_b200.so")

ABI_VERSION = 1
SUCCESS, INVALID_ARGUMENT, OUT_OF_MEMORY, CUDA_ERROR, INTERNAL_ERROR = range(5)
HOST, DEVICE = 0, 1
FIX_BRANCHING, FIX_BORDERS, FILTER_OBJECTS, DEVICE_OUTPUT, FILL_HOLES, FIX_AVOCADOS = 1, 2, 4, 8, 16, 32

DTYPES = {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.uint32): 2, np.dtype(np.uint64): 3,
          np.dtype(np.int8): 4, np.dtype(np.int16): 5, np.dtype(np.int32): 6, np.dtype(np.int64): 7,
          np.dtype(np.float32): 8, np.dtype(np.float64): 9}
DTYPE_NAMES = {v: k for k, v in DTYPES.items()}

# Every symbol include/brook_b200.h declares (the CPU tests check the library exports them all).
EXPORTS = ["brook_abi_version", "brook_version", "brook_last_error", "brook_context_create", "brook_context_destroy",
           "brook_context_synchronize", "brook_array_destroy", "brook_array_view", "brook_array_copy_to_host",
           "brook_connected_components", "brook_components_destroy", "brook_components_view",
           "brook_components_copy_to_host", "brook_edt", "brook_skeletonize_options_init", "brook_skeletonize",
           "brook_skeletonize_batch", "brook_skeletons_get_view", "brook_skeletons_destroy", "brook_context_stats",
           "brook_edt_device_noalloc", "brook_skeletons_get_device_view", "brook_skeletons_get_array",
           "brook_array_upload", "brook_array_to_dlpack", "brook_array_to_dlpack_versioned", "brook_components_labels",
           "brook_skeletonize_batch_targets", "brook_context_wait_stream", "brook_autotune",
           "brook_context_set_tuning", "brook_skeletons_create", "brook_merge_skeletons", "brook_context_trim",
           "brook_context_set_engine_share", "brook_postprocess_canonical", "brook_postprocess_step",
           "brook_skeleton_components", "brook_skeletons_create_device", "brook_connected_components_streamed",
           "brook_host_components_destroy", "brook_host_components_view", "brook_skeletonize_streamed",
           "brook_edt_streamed", "brook_pdrf_values"]


class Volume(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_size_t), ("abi_version", ctypes.c_uint32), ("data", ctypes.c_void_p),
                ("shape", ctypes.c_int64 * 3), ("strides", ctypes.c_int64 * 3), ("dtype", ctypes.c_int),
                ("memory", ctypes.c_int)]


class Teasar(ctypes.Structure):
    _fields_ = [("scale", ctypes.c_double), ("constant", ctypes.c_double), ("pdrf_scale", ctypes.c_double),
                ("pdrf_exponent", ctypes.c_double), ("soma_detection_threshold", ctypes.c_double),
                ("soma_acceptance_threshold", ctypes.c_double), ("soma_invalidation_scale", ctypes.c_double),
                ("soma_invalidation_const", ctypes.c_double), ("max_paths", ctypes.c_int64),
                ("has_max_paths", ctypes.c_uint32)]


class Options(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_size_t), ("abi_version", ctypes.c_uint32), ("teasar", Teasar),
                ("anisotropy", ctypes.c_float * 3), ("dust_threshold", ctypes.c_double), ("flags", ctypes.c_uint32),
                ("object_ids", ctypes.POINTER(ctypes.c_int64)), ("object_ids_count", ctypes.c_size_t),
                ("targets_before", ctypes.POINTER(ctypes.c_int64)), ("targets_before_count", ctypes.c_size_t),
                ("targets_after", ctypes.POINTER(ctypes.c_int64)), ("targets_after_count", ctypes.c_size_t),
                ("voxel_graph", ctypes.POINTER(Volume))]


class SkeletonsView(ctypes.Structure):
    _fields_ = [("skeleton_count", ctypes.c_size_t), ("vertex_count", ctypes.c_size_t), ("edge_count", ctypes.c_size_t),
                ("labels", ctypes.POINTER(ctypes.c_int64)), ("vertex_offsets", ctypes.POINTER(ctypes.c_int64)),
                ("edge_offsets", ctypes.POINTER(ctypes.c_int64)), ("vertices", ctypes.POINTER(ctypes.c_float)),
                ("edges", ctypes.POINTER(ctypes.c_uint32)), ("radii", ctypes.POINTER(ctypes.c_float)),
                ("anisotropy", ctypes.c_float * 3)]


class SkeletonsDeviceView(ctypes.Structure):
    _fields_ = [("skeleton_count", ctypes.c_size_t), ("vertex_count", ctypes.c_size_t), ("edge_count", ctypes.c_size_t),
                ("labels", ctypes.POINTER(ctypes.c_int64)), ("vertex_offsets", ctypes.POINTER(ctypes.c_int64)),
                ("edge_offsets", ctypes.POINTER(ctypes.c_int64)), ("vertices", Volume), ("edges", Volume),
                ("radii", Volume), ("anisotropy", ctypes.c_float * 3)]


class Tuning(ctypes.Structure):
    _fields_ = [("trace_cluster_ctas", ctypes.c_int32), ("trace_cluster_voxels", ctypes.c_int64),
                ("prepare_cluster_voxels", ctypes.c_int64), ("lone_first_percent", ctypes.c_int32)]


class SampleTargets(ctypes.Structure):
    _fields_ = [("before", ctypes.POINTER(ctypes.c_int64)), ("before_count", ctypes.c_size_t),
                ("after", ctypes.POINTER(ctypes.c_int64)), ("after_count", ctypes.c_size_t)]


VERTICES, EDGES, RADII = 0, 1, 2


class BrookError(RuntimeError):
    """A brook_b200 call failed; `status` is the brook_status code."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


_lib = None
_load_lock = threading.Lock()


def load():
    """The library handle, loaded on first use."""
    global _lib
    if _lib is None:
        with _load_lock:
            if _lib is None:
                _lib = _open()
    return _lib


def __getattr__(name):  # `_native.lib` loads the library on first use
    if name == "lib":
        return load()
    raise AttributeError(name)


def _open():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"brook_b200: the CUDA library {LIB_PATH} is not built; run brook_b200/build.py "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    sig = {
        "brook_abi_version": (ctypes.c_uint32, []),
        "brook_version": (ctypes.c_char_p, []),
        "brook_last_error": (ctypes.c_char_p, []),
        "brook_context_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(vp)]),
        "brook_context_destroy": (None, [vp]),
        "brook_context_synchronize": (ctypes.c_int, [vp]),
        "brook_context_trim": (ctypes.c_int, [vp]),
        "brook_context_set_engine_share": (ctypes.c_int, [vp, ctypes.c_int]),
        "brook_array_destroy": (None, [vp]),
        "brook_array_view": (ctypes.c_int, [vp, ctypes.POINTER(Volume)]),
        "brook_array_copy_to_host": (ctypes.c_int, [vp, vp, sz]),
        "brook_connected_components": (ctypes.c_int, [vp, ctypes.POINTER(Volume), ctypes.POINTER(vp)]),
        "brook_components_destroy": (None, [vp]),
        "brook_components_view": (ctypes.c_int, [vp, ctypes.POINTER(Volume), ctypes.POINTER(ctypes.POINTER(ctypes.c_int64)),
                                                 ctypes.POINTER(ctypes.POINTER(ctypes.c_int64)), ctypes.POINTER(sz)]),
        "brook_components_copy_to_host": (ctypes.c_int, [vp, vp, sz]),
        "brook_edt": (ctypes.c_int, [vp, ctypes.POINTER(Volume), ctypes.POINTER(ctypes.c_float), ctypes.c_int,
                                     ctypes.POINTER(vp)]),
        "brook_skeletonize_options_init": (None, [ctypes.POINTER(Options)]),
        "brook_skeletonize": (ctypes.c_int, [vp, ctypes.POINTER(Volume), ctypes.POINTER(Options), ctypes.POINTER(vp)]),
        "brook_skeletonize_batch": (ctypes.c_int, [vp, ctypes.POINTER(Volume), sz, ctypes.POINTER(Options),
                                                   ctypes.POINTER(vp)]),
        "brook_skeletons_get_view": (ctypes.c_int, [vp, ctypes.POINTER(SkeletonsView)]),
        "brook_skeletons_destroy": (None, [vp]),
        "brook_context_stats": (ctypes.c_int, [vp, ctypes.c_char_p, sz, ctypes.POINTER(sz)]),
        "brook_edt_device_noalloc": (ctypes.c_int, [ctypes.POINTER(Volume), ctypes.POINTER(ctypes.c_float), ctypes.c_int,
                                                    vp, vp]),
        "brook_skeletons_get_device_view": (ctypes.c_int, [vp, ctypes.POINTER(SkeletonsDeviceView)]),
        "brook_skeletons_get_array": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(vp)]),
        "brook_array_upload": (ctypes.c_int, [vp, ctypes.POINTER(Volume), ctypes.POINTER(vp)]),
        "brook_array_to_dlpack": (ctypes.c_int, [vp, ctypes.POINTER(vp)]),
        "brook_array_to_dlpack_versioned": (ctypes.c_int, [vp, ctypes.c_uint32, ctypes.POINTER(vp)]),
        "brook_components_labels": (ctypes.c_int, [vp, ctypes.POINTER(vp)]),
        "brook_skeletonize_batch_targets": (ctypes.c_int, [vp, ctypes.POINTER(Volume), sz, ctypes.POINTER(Options),
                                                           ctypes.POINTER(SampleTargets), ctypes.POINTER(vp)]),
        "brook_context_wait_stream": (ctypes.c_int, [vp, ctypes.c_int64]),
        "brook_autotune": (ctypes.c_int, [vp, ctypes.POINTER(Volume), sz, ctypes.POINTER(Options),
                                          ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(Tuning),
                                          ctypes.POINTER(ctypes.c_double)]),
        "brook_context_set_tuning": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.POINTER(Tuning)]),
        "brook_skeletons_create": (ctypes.c_int, [ctypes.POINTER(SkeletonsView), ctypes.POINTER(vp)]),
        "brook_merge_skeletons": (ctypes.c_int, [vp, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_float), sz,
                                                 ctypes.POINTER(vp)]),
        "brook_postprocess_canonical": (ctypes.c_int, [vp, vp, ctypes.c_double, ctypes.c_double, ctypes.POINTER(vp)]),
        "brook_postprocess_step": (ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.c_double, ctypes.POINTER(vp)]),
        "brook_skeleton_components": (ctypes.c_int, [vp, vp, ctypes.POINTER(vp)]),
        "brook_skeletons_create_device": (ctypes.c_int, [vp, ctypes.POINTER(SkeletonsDeviceView), ctypes.POINTER(vp)]),
        "brook_connected_components_streamed": (ctypes.c_int, [vp, ctypes.POINTER(Volume), sz, ctypes.POINTER(vp)]),
        "brook_host_components_destroy": (None, [vp]),
        "brook_host_components_view": (ctypes.c_int, [vp, ctypes.POINTER(Volume),
                                                      ctypes.POINTER(ctypes.POINTER(ctypes.c_int64)),
                                                      ctypes.POINTER(ctypes.POINTER(ctypes.c_int64)),
                                                      ctypes.POINTER(sz)]),
        "brook_skeletonize_streamed": (ctypes.c_int, [vp, ctypes.POINTER(Volume), ctypes.POINTER(Options), sz,
                                                      ctypes.POINTER(vp)]),
        "brook_edt_streamed": (ctypes.c_int, [vp, ctypes.POINTER(Volume), ctypes.POINTER(ctypes.c_float), ctypes.c_int,
                                              sz, vp, sz]),
        "brook_pdrf_values": (ctypes.c_int, [vp, vp, vp, sz, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def check(status):
    if status != SUCCESS:
        raise BrookError(status, load().brook_last_error().decode(errors="replace"))


class _ThreadContexts(dict):
    """One thread's contexts by (process, device). Held in a threading.local, so it is released
    when its thread ends, and every context it holds (streams, kept device blocks, the engine's
    executable graph) is destroyed with it."""

    def __del__(self):
        lib = _lib
        if lib is None:
            return
        for (pid, _), handle in self.items():
            if pid == os.getpid():
                try:
                    lib.brook_context_destroy(handle)
                except Exception:  # interpreter shutdown
                    pass
        self.clear()


_local = threading.local()


def context(device=0):
    """One context per (process, thread, device), as the reference's runtime keeps them; a thread's
    contexts are destroyed when the thread ends."""
    contexts = getattr(_local, "contexts", None)
    if contexts is None:
        contexts = _local.contexts = _ThreadContexts()
    key = (os.getpid(), int(device))
    ctx = contexts.get(key)
    if ctx is None:
        handle = ctypes.c_void_p()
        check(load().brook_context_create(int(device), ctypes.byref(handle)))
        ctx = contexts[key] = handle
        from . import tuning

        tuning.install_saved(handle, int(device))
    return ctx


def host_volume(array):
    """A brook_volume over a NumPy array (any strides); the array must outlive the call."""
    v = Volume()
    v.struct_size = ctypes.sizeof(Volume)
    v.abi_version = ABI_VERSION
    v.data = array.ctypes.data if array.size else None
    for a in range(3):
        v.shape[a] = array.shape[a]
        v.strides[a] = array.strides[a]
    v.dtype = DTYPES[array.dtype]
    v.memory = HOST
    return v


def device_volume(ptr, shape, strides_bytes, dtype):
    v = Volume()
    v.struct_size = ctypes.sizeof(Volume)
    v.abi_version = ABI_VERSION
    v.data = ptr
    for a in range(3):
        v.shape[a] = shape[a]
        v.strides[a] = strides_bytes[a]
    v.dtype = DTYPES[np.dtype(dtype)]
    v.memory = DEVICE
    return v


def options(teasar, anisotropy, dust_threshold, fix_branching, fix_borders, object_ids=None,
            targets_before=(), targets_after=()):
    o = Options()
    load().brook_skeletonize_options_init(ctypes.byref(o))
    t = o.teasar
    t.scale, t.constant, t.pdrf_scale, t.pdrf_exponent = (teasar["scale"], teasar["const"], teasar["pdrf_scale"],
                                                          teasar["pdrf_exponent"])
    t.soma_detection_threshold = teasar["soma_detection_threshold"]
    t.soma_acceptance_threshold = teasar["soma_acceptance_threshold"]
    t.soma_invalidation_scale = teasar["soma_invalidation_scale"]
    t.soma_invalidation_const = teasar["soma_invalidation_const"]
    if teasar.get("max_paths") is not None:
        t.max_paths, t.has_max_paths = int(teasar["max_paths"]), 1
    o.anisotropy[:] = [float(a) for a in anisotropy]
    o.dust_threshold = float(dust_threshold)
    o.flags = (FIX_BRANCHING if fix_branching else 0) | (FIX_BORDERS if fix_borders else 0)
    keep = []
    if object_ids is not None:
        ids = np.ascontiguousarray(np.asarray(list(object_ids), dtype=np.int64))
        keep.append(ids)
        o.flags |= FILTER_OBJECTS
        o.object_ids = ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        o.object_ids_count = ids.size
    for name, points in (("targets_before", targets_before), ("targets_after", targets_after)):
        pts = np.ascontiguousarray(np.asarray(list(points), dtype=np.int64).reshape(-1, 3))
        if pts.size:
            keep.append(pts)
            setattr(o, name, pts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
            setattr(o, name + "_count", pts.shape[0])
    o._keep = keep  # the arrays the pointers refer to
    return o


def packed_arrays(handle):
    """Copies a brook_skeletons result into NumPy arrays and releases the handle."""
    v = SkeletonsView()
    try:
        check(load().brook_skeletons_get_view(handle, ctypes.byref(v)))

        def grab(ptr, count, dtype, shape):
            if count == 0:
                return np.zeros(shape, dtype)
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dtype, copy=True).reshape(shape)

        k, nv, ne = v.skeleton_count, v.vertex_count, v.edge_count
        return dict(labels=grab(v.labels, k, np.int64, (k,)), v_off=grab(v.vertex_offsets, k + 1, np.int64, (k + 1,)),
                    e_off=grab(v.edge_offsets, k + 1, np.int64, (k + 1,)),
                    vertices=grab(v.vertices, 3 * nv, np.float32, (nv, 3)), edges=grab(v.edges, 2 * ne, np.uint32, (ne, 2)),
                    radii=grab(v.radii, nv, np.float32, (nv,)), anisotropy=tuple(float(a) for a in v.anisotropy))
    finally:
        load().brook_skeletons_destroy(handle)


class _DeviceResult:
    """Owns a brook_skeletons device result; its arrays are exposed without copies (CUDA array
    interface) and the result is destroyed when the last array viewing it goes away."""

    def __init__(self, handle):
        self.handle = handle

    def __del__(self):
        if self.handle:
            load().brook_skeletons_destroy(self.handle)
            self.handle = None


class _DeviceArray:
    def __init__(self, owner, ptr, shape, typestr):
        self.owner = owner  # keeps the result alive
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (int(ptr or 0), False),
                                         "version": 3, "strides": None}


def packed_device_arrays(handle):
    """A BROOK_DEVICE_OUTPUT result as host metadata and torch CUDA tensors over the result's own
    device arrays (no copy); the handle lives as long as those tensors."""
    import torch

    v = SkeletonsDeviceView()
    owner = _DeviceResult(handle)
    check(load().brook_skeletons_get_device_view(handle, ctypes.byref(v)))
    k, nv, ne = v.skeleton_count, v.vertex_count, v.edge_count

    def host(ptr, count):
        return np.ctypeslib.as_array(ptr, shape=(count,)).astype(np.int64, copy=True) if count else np.zeros(0, np.int64)

    def device(vol, shape, typestr, dtype):
        if not np.prod(shape):
            return torch.zeros(shape, dtype=dtype, device="cuda")
        return torch.as_tensor(_DeviceArray(owner, vol.data, shape, typestr), device="cuda")

    return dict(labels=host(v.labels, k), v_off=host(v.vertex_offsets, k + 1), e_off=host(v.edge_offsets, k + 1),
                vertices=device(v.vertices, (nv, 3), "<f4", torch.float32),
                edges=device(v.edges, (ne, 2), "<u4", torch.uint32),
                radii=device(v.radii, (nv,), "<f4", torch.float32),
                anisotropy=tuple(float(a) for a in v.anisotropy))


def skeletons_handle(packed, device=0):
    """A new brook_skeletons handle holding a copy of PackedSkeletons: host arrays through
    brook_skeletons_create, CUDA tensors through brook_skeletons_create_device (on the device,
    ordered after the current torch stream). The caller destroys it."""
    lib = load()
    h = ctypes.c_void_p()
    if not packed.on_device:
        p = packed
        keep = [np.ascontiguousarray(p.labels, np.int64), np.ascontiguousarray(p.v_off, np.int64),
                np.ascontiguousarray(p.e_off, np.int64), np.ascontiguousarray(p.vertices, np.float32).reshape(-1, 3),
                np.ascontiguousarray(p.edges, np.uint32).reshape(-1, 2), np.ascontiguousarray(p.radii, np.float32)]
        v = SkeletonsView()
        v.skeleton_count, v.vertex_count, v.edge_count = len(keep[0]), len(keep[5]), len(keep[4])
        v.labels = keep[0].ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        v.vertex_offsets = keep[1].ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        v.edge_offsets = keep[2].ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        v.vertices = keep[3].ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        v.edges = keep[4].ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        v.radii = keep[5].ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        v.anisotropy[:] = [float(x) for x in p.anisotropy]
        check(lib.brook_skeletons_create(ctypes.byref(v), ctypes.byref(h)))
        return h.value
    import torch

    ctx = context(device)
    check(lib.brook_context_wait_stream(ctx, torch.cuda.current_stream(device).cuda_stream))
    tensors = [packed.vertices.contiguous(), packed.edges.contiguous(), packed.radii.contiguous()]
    meta = [np.ascontiguousarray(packed.labels, np.int64), np.ascontiguousarray(packed.v_off, np.int64),
            np.ascontiguousarray(packed.e_off, np.int64)]
    v = SkeletonsDeviceView()
    v.skeleton_count, v.vertex_count, v.edge_count = len(meta[0]), int(meta[1][-1]), int(meta[2][-1])
    v.labels = meta[0].ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    v.vertex_offsets = meta[1].ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    v.edge_offsets = meta[2].ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    for field, t, width, code in ((v.vertices, tensors[0], 3, 8), (v.edges, tensors[1], 2, 2), (v.radii, tensors[2], 1, 8)):
        rows = t.numel() // width
        field.struct_size, field.abi_version = ctypes.sizeof(Volume), ABI_VERSION
        field.data = t.data_ptr() if rows else None
        field.shape[:] = [width, rows, 1]
        field.strides[:] = [4, 4 * width, 4 * width * rows]
        field.dtype, field.memory = code, DEVICE
    v.anisotropy[:] = [float(x) for x in packed.anisotropy]
    check(lib.brook_skeletons_create_device(ctx, ctypes.byref(v), ctypes.byref(h)))
    return h.value


def array_tensor(array_handle):
    """A brook_array as a torch tensor over its own device memory (DLPack, no copy); the array
    handle is released (the export keeps the memory alive)."""
    import torch

    lib = load()
    dl = ctypes.c_void_p()
    try:
        check(lib.brook_array_to_dlpack(array_handle, ctypes.byref(dl)))
    finally:
        lib.brook_array_destroy(array_handle)
    make = ctypes.pythonapi.PyCapsule_New
    make.restype = ctypes.py_object
    make.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
    return torch.utils.dlpack.from_dlpack(make(dl.value, b"dltensor", None))


def trim(device=0):
    """Returns the device memory the calling thread's context keeps for reuse to the driver."""
    check(load().brook_context_trim(context(device)))


def set_engine_share(percent, device=0):
    """The share (percent) of the GPU's resident clusters the calling thread's context's
    persistent engine launches take (brook_context_set_engine_share)."""
    check(load().brook_context_set_engine_share(context(device), int(percent)))


def stats(device=0):
    """The statistics of the calling thread's context's last call (stage ms and work counters)."""
    import json

    ctx = context(device)
    need = ctypes.c_size_t()
    check(load().brook_context_stats(ctx, None, 0, ctypes.byref(need)))
    buf = ctypes.create_string_buffer(need.value)
    check(load().brook_context_stats(ctx, buf, need.value, None))
    return json.loads(buf.value.decode())
