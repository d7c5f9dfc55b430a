"""CPU restatement of the reference's canonical post-processing of packed skeletons
(brook_postprocess_canonical, cpp/include/brook/brook.h:238-239; cpp/src/post.cu:646-650 and
cpp/src/post_kernels.cuh), implemented in oracle/post.cpp.

TEST INFRASTRUCTURE ONLY: the checker of brook_b200's device post-processing; the product never
imports it.

A packed set is a dict of arrays: labels (K,), vertex_offsets (K+1,), edge_offsets (K+1,),
vertices (V, 3) float32, edges (E, 2) uint32 local to each skeleton, radii (V,) float32.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import oracle as _oracle

STEPS = {"postprocess": 0, "remove_dust": 1, "remove_loops": 2, "join_components": 3, "remove_ticks": 4,
         "prune_unused": 5, "components": 6}


def _lib():
    lib = _oracle.lib()
    if not getattr(lib, "_post_ready", False):
        p = ctypes.c_void_p
        lib.oracle_post.restype = p
        lib.oracle_post.argtypes = [p, ctypes.c_int64, p, p, p, p, p, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        lib.oracle_post_error.restype = ctypes.c_char_p
        lib.oracle_post_error.argtypes = [p]
        lib.oracle_post_sizes.argtypes = [p, p]
        lib.oracle_post_copy.argtypes = [p, p, p, p, p, p, p, p]
        lib.oracle_post_free.argtypes = [p]
        lib._post_ready = True
    return lib


def _arrays(packed):
    labels = np.ascontiguousarray(packed["labels"], np.int64)
    voff = np.ascontiguousarray(packed["vertex_offsets"], np.int64)
    eoff = np.ascontiguousarray(packed["edge_offsets"], np.int64)
    vertices = np.ascontiguousarray(np.asarray(packed["vertices"], np.float32).reshape(-1, 3))
    edges = np.ascontiguousarray(np.asarray(packed["edges"], np.uint32).reshape(-1, 2))
    radii = np.ascontiguousarray(packed["radii"], np.float32)
    return labels, voff, eoff, vertices, edges, radii


def run(packed, step, a=0.0, b=0.0):
    """One step ("postprocess" with a = dust and b = tick threshold, "remove_dust" / "remove_ticks"
    with a = threshold, "remove_loops", "join_components", "prune_unused") -> a packed dict;
    "components" -> the int64 component id (smallest vertex id) of every vertex."""
    lib = _lib()
    arrays = _arrays(packed)
    ptr = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    h = lib.oracle_post(ptr(arrays[0]), len(arrays[0]), *[ptr(x) for x in arrays[1:]], STEPS[step], float(a), float(b))
    try:
        err = lib.oracle_post_error(h)
        if err:
            raise ValueError(err.decode())
        sizes = np.zeros(4, np.int64)
        lib.oracle_post_sizes(h, ptr(sizes))
        k, nv, ne, nc = (int(s) for s in sizes)
        out = dict(labels=np.zeros(k, np.int64), vertex_offsets=np.zeros(k + 1, np.int64),
                   edge_offsets=np.zeros(k + 1, np.int64), vertices=np.zeros((nv, 3), np.float32),
                   edges=np.zeros((ne, 2), np.uint32), radii=np.zeros(nv, np.float32))
        comps = np.zeros(nc, np.int64)
        lib.oracle_post_copy(h, *[ptr(out[n]) for n in ("labels", "vertex_offsets", "edge_offsets", "vertices",
                                                         "edges", "radii")], ptr(comps))
    finally:
        lib.oracle_post_free(h)
    return comps if step == "components" else out


def postprocess(packed, dust_threshold=1500, tick_threshold=3500):
    return run(packed, "postprocess", dust_threshold, tick_threshold)
