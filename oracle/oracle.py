"""ctypes wrapper of the CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline, always as the checker. The product package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_DTYPES = {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.uint32): 2, np.dtype(np.uint64): 3,
           np.dtype(np.int8): 4, np.dtype(np.int16): 5, np.dtype(np.int32): 6, np.dtype(np.int64): 7}


class _Params(ctypes.Structure):
    _fields_ = [("scale", ctypes.c_double), ("constant", ctypes.c_double), ("pdrf_scale", ctypes.c_double),
                ("pdrf_exponent", ctypes.c_double), ("soma_detection", ctypes.c_double),
                ("soma_acceptance", ctypes.c_double), ("soma_scale", ctypes.c_double),
                ("soma_constant", ctypes.c_double), ("max_paths", ctypes.c_int64), ("has_max_paths", ctypes.c_int32),
                ("anisotropy", ctypes.c_float * 3), ("dust", ctypes.c_double), ("fix_branching", ctypes.c_int32),
                ("fix_borders", ctypes.c_int32), ("targets_before", ctypes.POINTER(ctypes.c_int64)),
                ("n_before", ctypes.c_int64), ("targets_after", ctypes.POINTER(ctypes.c_int64)),
                ("n_after", ctypes.c_int64), ("pdrf_field", ctypes.POINTER(ctypes.c_float)),
                ("fill_holes", ctypes.c_int32), ("fix_avocados", ctypes.c_int32)]


_lib = None


def build():
    """Compile the oracle (a few seconds with g++)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        newest = max(os.path.getmtime(os.path.join(_HERE, f)) for f in ("oracle.cpp", "post.cpp", "graph.cpp"))
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < newest:
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.oracle_run.restype = ctypes.c_void_p
        _lib.oracle_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                    ctypes.POINTER(_Params), ctypes.c_int, ctypes.c_int]
        _lib.oracle_free.argtypes = [ctypes.c_void_p]
        _lib.oracle_error.restype = ctypes.c_char_p
        _lib.oracle_error.argtypes = [ctypes.c_void_p]
        _lib.oracle_array.restype = ctypes.c_void_p
        _lib.oracle_array.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
        _lib.oracle_borders.restype = ctypes.c_int64
        _lib.oracle_borders.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64]
        _lib.oracle_edt.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        _lib.oracle_railroad_graph.restype = ctypes.c_int64
        _lib.oracle_railroad_graph.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                               ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
                                               ctypes.c_int64]
        _lib.oracle_railroad.restype = ctypes.c_int64
        _lib.oracle_railroad.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                         ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64]
        _lib.oracle_railroad_distances.restype = ctypes.c_int
        _lib.oracle_railroad_distances.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                                   ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p]
        _lib.oracle_pyset.restype = ctypes.c_int64
        _lib.oracle_pyset.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64]
        _lib.oracle_target_order.restype = ctypes.c_int64
        _lib.oracle_target_order.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
        _lib.oracle_prepare.restype = ctypes.c_void_p
        _lib.oracle_prepare.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                        ctypes.POINTER(_Params), ctypes.c_int]
        _lib.oracle_objects.restype = ctypes.c_int64
        _lib.oracle_objects.argtypes = [ctypes.c_void_p]
        _lib.oracle_trace.restype = ctypes.c_int
        _lib.oracle_trace.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int]
        _lib.oracle_finish.restype = ctypes.c_int
        _lib.oracle_finish.argtypes = [ctypes.c_void_p]
    return _lib


# kimimaro.trace defaults for teasar keys a caller leaves out (the reference's TraceParameters,
# skeleton.hpp:23-27)
TRACE_DEFAULTS = dict(scale=10.0, const=10.0, pdrf_scale=5000.0, pdrf_exponent=16.0, soma_detection_threshold=1100.0,
                      soma_acceptance_threshold=4000.0, soma_invalidation_scale=0.5, soma_invalidation_const=0.0)

_ARRAY_TYPES = {"labels": np.int64, "vertex_offsets": np.int64, "edge_offsets": np.int64, "vertices": np.float32,
                "radii": np.float32, "edges": np.uint32, "cc": np.uint32, "mapping": np.int64, "cc_roots": np.int64,
                "dbf": np.float32, "daf": np.float32, "pdrf": np.float32, "roots": np.int64, "targets": np.int64,
                "boxes": np.int64, "orders": np.int64, "order_offsets": np.int64, "paths": np.int64,
                "path_offsets": np.int64, "path_labels": np.int64, "stage_ms": np.float64,
                "filled": np.int64, "avocado_passes": np.int64}

# names of the entries of OracleResult.array("stage_ms"): wall-clock ms of each step
STAGES = ("components", "boxes", "edt", "borders", "daf", "pdrf", "orders", "trace", "assembly")


class OracleResult:
    """Packed skeletons and (with stages=True) the intermediate fields of one oracle run."""

    def __init__(self, handle, shape):
        self._h = handle
        self.shape = shape

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.oracle_free(self._h)
            self._h = None

    def stage_ms(self):
        """{step: wall-clock ms} of the run."""
        return dict(zip(STAGES, self.array("stage_ms").tolist()))

    def array(self, name):
        count = ctypes.c_int64(0)
        ptr = lib().oracle_array(self._h, name.encode(), ctypes.byref(count))
        dtype = np.dtype(_ARRAY_TYPES[name])
        if count.value <= 0:
            return np.zeros(0, dtype)
        buf = (ctypes.c_char * (count.value * dtype.itemsize)).from_address(ptr)
        return np.frombuffer(buf, dtype).copy()

    def field(self, name):
        return self.array(name).reshape(self.shape, order="F")

    def borders(self, component_id):
        out = np.zeros(3 * 4096, np.int64)
        n = lib().oracle_borders(self._h, component_id, out.ctypes.data, out.size)
        return [tuple(int(v) for v in out[3 * i:3 * i + 3]) for i in range(max(n, 0))]

    def packed(self):
        return dict(labels=self.array("labels"), vertex_offsets=self.array("vertex_offsets"),
                    edge_offsets=self.array("edge_offsets"), vertices=self.array("vertices").reshape(-1, 3),
                    edges=self.array("edges").reshape(-1, 2), radii=self.array("radii"))

    def skeletons(self):
        """{label: (vertices float32 (V,3), edges uint32 (E,2), radii float32 (V,))}"""
        p = self.packed()
        out = {}
        for k, label in enumerate(p["labels"].tolist()):
            v0, v1 = int(p["vertex_offsets"][k]), int(p["vertex_offsets"][k + 1])
            e0, e1 = int(p["edge_offsets"][k]), int(p["edge_offsets"][k + 1])
            out[int(label)] = (p["vertices"][v0:v1], p["edges"][e0:e1], p["radii"][v0:v1])
        return out


def _params(teasar_params, anisotropy, dust_threshold, fix_branching, fix_borders):
    t = dict(TRACE_DEFAULTS)
    max_paths = None
    for key, value in dict(teasar_params).items():
        if key == "max_paths":
            max_paths = value
        elif key not in t:
            raise TypeError(f"unexpected TEASAR parameter: {key}")
        else:
            t[key] = float(value)
    p = _Params()
    p.scale, p.constant, p.pdrf_scale, p.pdrf_exponent = t["scale"], t["const"], t["pdrf_scale"], t["pdrf_exponent"]
    p.soma_detection, p.soma_acceptance = t["soma_detection_threshold"], t["soma_acceptance_threshold"]
    p.soma_scale, p.soma_constant = t["soma_invalidation_scale"], t["soma_invalidation_const"]
    p.max_paths, p.has_max_paths = (0, 0) if max_paths is None else (int(max_paths), 1)
    p.anisotropy[:] = [float(a) for a in anisotropy]
    p.dust = float(dust_threshold)
    p.fix_branching, p.fix_borders = int(bool(fix_branching)), int(bool(fix_borders))
    return p


# The teasar_params default of the reference's brook.skeletonize (src/brook/__init__.py:8-17).
DEFAULT_TEASAR_PARAMS = dict(scale=1.5, const=300, pdrf_scale=100000, pdrf_exponent=4, soma_acceptance_threshold=3500,
                             soma_detection_threshold=750, soma_invalidation_const=300, soma_invalidation_scale=2)


def skeletonize(labels, teasar_params=DEFAULT_TEASAR_PARAMS, anisotropy=(1, 1, 1), dust_threshold=1000,
                fix_branching=True, fix_borders=True, threads=1, stages=False, extra_targets_before=(),
                extra_targets_after=(), pdrf_field=None, fill_holes=False, fix_avocados=False):
    """Run the oracle on a 3D label volume (any layout; read as its logical (x, y, z) axes), with
    the argument defaults of the reference's brook.skeletonize. `pdrf_field` (float32, the
    volume's shape) replaces the oracle's own PDRF over the traced objects: a test traces from
    another implementation's field where the power itself is not bit-reproducible (an exponent
    that is not a power of two). With `fill_holes`, array("filled") holds the voxels filled; with
    `fix_avocados`, array("avocado_passes") the avocado stage's passes."""
    labels = np.asarray(labels)
    if labels.dtype == bool:
        labels = labels.view(np.uint8)
    while labels.ndim < 3:
        labels = labels[..., np.newaxis]
    labels = np.asfortranarray(labels)
    if labels.dtype not in _DTYPES:
        raise TypeError(f"unsupported label dtype {labels.dtype}")
    params = _params(teasar_params or {}, anisotropy, dust_threshold, fix_branching, fix_borders)
    params.fill_holes = int(bool(fill_holes))
    params.fix_avocados = int(bool(fix_avocados))
    keep = []
    for name, points in (("targets_before", extra_targets_before), ("targets_after", extra_targets_after)):
        pts = np.ascontiguousarray(np.asarray(list(points), np.int64).reshape(-1, 3))
        keep.append(pts)
        setattr(params, name, pts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        setattr(params, "n_before" if name == "targets_before" else "n_after", pts.shape[0])
    if pdrf_field is not None:
        field = np.asfortranarray(np.asarray(pdrf_field, np.float32))
        if field.shape != labels.shape:
            raise ValueError("pdrf_field must have the volume's shape")
        keep.append(field)
        params.pdrf_field = field.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    handle = lib().oracle_run(labels.ctypes.data, _DTYPES[labels.dtype], *labels.shape, ctypes.byref(params),
                              int(threads), int(bool(stages)))
    result = OracleResult(handle, labels.shape)
    error = lib().oracle_error(handle).decode()
    if error:
        raise RuntimeError(f"oracle: {error}")
    return result


class StagedRun:
    """The oracle's path in steps over one volume: prepare() on construction, trace(begin, end)
    over sub-ranges of the largest-first object order (`objects` of them), finish() for the
    packed result. Lets a caller spread one volume's work over several timed steps."""

    def __init__(self, labels, teasar_params=DEFAULT_TEASAR_PARAMS, anisotropy=(1, 1, 1), dust_threshold=1000,
                 fix_branching=True, fix_borders=True, threads=1):
        labels = np.asfortranarray(np.asarray(labels))
        self.shape = labels.shape
        self._labels = labels
        self.params = _params(teasar_params or {}, anisotropy, dust_threshold, fix_branching, fix_borders)
        self.threads = int(threads)
        self.result = OracleResult(lib().oracle_prepare(labels.ctypes.data, _DTYPES[labels.dtype], *labels.shape,
                                                        ctypes.byref(self.params), self.threads), labels.shape)
        self._check()
        self.objects = int(lib().oracle_objects(self.result._h))

    def _check(self):
        error = lib().oracle_error(self.result._h).decode()
        if error:
            raise RuntimeError(f"oracle: {error}")

    def trace(self, begin, end):
        if lib().oracle_trace(self.result._h, int(begin), int(end), self.threads):
            self._check()

    def finish(self):
        if lib().oracle_finish(self.result._h):
            self._check()
        return self.result


def edt(labels, anisotropy=(1, 1, 1), black_border=False, dims=3):
    labels = np.asfortranarray(np.asarray(labels, np.uint32))
    while labels.ndim < 3:
        labels = labels[..., np.newaxis]
    out = np.zeros(labels.shape, np.float32, order="F")
    aniso = np.asarray(anisotropy, np.float32)
    if lib().oracle_edt(labels.ctypes.data, *labels.shape, aniso.ctypes.data, int(bool(black_border)), int(dims),
                        out.ctypes.data):
        raise RuntimeError("oracle EDT failed")
    return out


def railroad(field, target, component=None, voxel_graph=None):
    """The railroad path (target first) over `component` (default: every voxel); `voxel_graph`:
    cc3d bits per voxel that gate every step (oracle_railroad_graph)."""
    field = np.asfortranarray(np.asarray(field, np.float32))
    comp = np.ones(field.shape, np.uint32, order="F") if component is None else np.asfortranarray(component.astype(np.uint32))
    out = np.zeros(field.size, np.int64)
    graph = None if voxel_graph is None else np.asfortranarray(np.asarray(voxel_graph, np.uint32))
    if graph is not None and graph.shape != field.shape:
        raise ValueError("voxel_graph must match the field")
    n = lib().oracle_railroad_graph(field.ctypes.data, comp.ctypes.data, None if graph is None else graph.ctypes.data,
                                    *field.shape, int(target), out.ctypes.data, out.size)
    return out[:n].tolist()


def railroad_distances(field, target, component=None):
    """The railroad's float32 distance field from `target` (+inf where the search never reached)."""
    field = np.asfortranarray(np.asarray(field, np.float32))
    comp = np.ones(field.shape, np.uint32, order="F") if component is None else np.asfortranarray(component.astype(np.uint32))
    out = np.zeros(field.shape, np.float32, order="F")
    if lib().oracle_railroad_distances(field.ctypes.data, comp.ctypes.data, *field.shape, int(target), out.ctypes.data):
        raise RuntimeError("oracle railroad failed")
    return out


def pyset_order(ops):
    """The iteration order of set A after a script of (code, key) operations (oracle_pyset)."""
    ops = np.ascontiguousarray(np.asarray(ops, np.int64).reshape(-1, 2))
    out = np.zeros(max(len(ops), 1), np.int64)
    n = lib().oracle_pyset(ops.ctypes.data, len(ops), out.ctypes.data, out.size)
    return out[:n].tolist()


def target_order(mask, daf):
    mask = np.ascontiguousarray(mask, np.uint8)
    daf = np.ascontiguousarray(daf, np.float32)
    out = np.zeros(mask.size, np.int64)
    n = lib().oracle_target_order(mask.ctypes.data, daf.ctypes.data, mask.size, out.ctypes.data)
    return out[:n]


def pdrf_values(dbf, daf, maximum, max_daf, scale, exponent):
    """The reference's PDRF arithmetic on arrays of DBF / DAF values (oracle_pdrf_values)."""
    l = lib()
    if not getattr(l, "_pdrf_ready", False):
        l.oracle_pdrf_values.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
        l._pdrf_ready = True
    dbf = np.ascontiguousarray(dbf, np.float32)
    daf = np.ascontiguousarray(daf, np.float32)
    out = np.empty_like(dbf)
    l.oracle_pdrf_values(dbf.ctypes.data, daf.ctypes.data, dbf.size, float(maximum), float(max_daf), float(scale),
                         float(exponent), out.ctypes.data)
    return out
