"""CPU restatement of the reference's voxel-graph preamble (oracle/graph.cpp): the components of
a voxel connectivity graph (brook_graph_components, cpp/src/c_api.cpp:201-207;
cpp/src/graph_components.cu) and the graph-aware EDT (brook_graph_edt, cpp/src/c_api.cpp:209-216;
cpp/src/graph_edt.cu).

TEST INFRASTRUCTURE ONLY: the checker for a device implementation of these calls; the product
never imports it.

Volumes are Fortran-ordered (x fastest). A graph is cc3d's uint32 bitfield per voxel (bit b
permits the step STEPS[b]) or its compact 2D uint8 form.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import oracle as _oracle

# cc3d's bit order: bit b permits the step STEPS[b] = (dx, dy, dz) along the array's own axes
STEPS = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
         (1, 1, 0), (-1, 1, 0), (1, -1, 0), (-1, -1, 0), (1, 0, 1), (-1, 0, 1),
         (0, 1, 1), (0, -1, 1), (1, 0, -1), (-1, 0, -1), (0, 1, -1), (0, -1, -1),
         (1, 1, 1), (-1, 1, 1), (1, -1, 1), (-1, -1, 1), (1, 1, -1), (-1, 1, -1),
         (1, -1, -1), (-1, -1, -1)]


def _lib():
    lib = _oracle.lib()
    if not getattr(lib, "_graph_ready", False):
        p, i64 = ctypes.c_void_p, ctypes.c_int64
        lib.oracle_graph_components.restype = i64
        lib.oracle_graph_components.argtypes = [p, p, ctypes.c_int, i64, i64, i64, p, p, p, p]
        lib.oracle_graph_edt.restype = ctypes.c_int
        lib.oracle_graph_edt.argtypes = [p, p, ctypes.c_int, i64, i64, i64, p, ctypes.c_int, p]
        lib._graph_ready = True
    return lib


def _inputs(labels, graph):
    labels = np.asarray(labels)
    while labels.ndim < 3:
        labels = labels[..., np.newaxis]
    graph = np.asarray(graph)
    while graph.ndim < 3:
        graph = graph[..., np.newaxis]
    if graph.shape != labels.shape or graph.dtype not in (np.uint8, np.uint32):
        raise ValueError("voxel_graph must be uint8 or uint32 and match the volume")
    return (np.asfortranarray(labels.astype(np.uint64, copy=False)), np.asfortranarray(graph),
            int(graph.dtype == np.uint8))


def graph_components(labels, graph):
    """-> (ids uint32 (0 for background), mapping (count + 1,), roots (count,), keys (count + 1,)):
    compact ids by each graph component's lowest voxel, the label at the start of each id's last
    run of voxels, each id's lowest voxel, each id's rank among all graph components (background
    ones included)."""
    labels, graph, u8 = _inputs(labels, graph)
    n = labels.size
    ids = np.zeros(labels.shape, np.uint32, order="F")
    mapping, roots, keys = (np.zeros(n + 1, np.int64) for _ in range(3))
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    count = _lib().oracle_graph_components(ptr(labels), ptr(graph), u8, *labels.shape, ptr(ids), ptr(mapping),
                                           ptr(roots), ptr(keys))
    if count < 0:
        raise ValueError("bad volume")
    return ids, mapping[:count + 1].copy(), roots[:count].copy(), keys[:count + 1].copy()


def graph_edt(labels, graph, anisotropy=(1, 1, 1), black_border=False):
    """The graph-aware EDT: blocked face interfaces at half a voxel (float32, 0 on background)."""
    labels, graph, u8 = _inputs(labels, graph)
    out = np.zeros(labels.shape, np.float32, order="F")
    aniso = np.asarray(anisotropy, np.float32)
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    if _lib().oracle_graph_edt(ptr(labels), ptr(graph), u8, *labels.shape, ptr(aniso), int(bool(black_border)),
                               ptr(out)):
        raise ValueError("bad volume or anisotropy")
    return out


def label_graph(labels):
    """Each voxel's permitted steps to an in-volume neighbour of the same label (background
    included): the graph under which graph components are the labels' own 26-connected components."""
    labels = np.asarray(labels)
    graph = np.zeros(labels.shape, np.uint32)
    for bit, (dx, dy, dz) in enumerate(STEPS):
        src = tuple(slice(max(0, -d), labels.shape[a] - max(0, d)) for a, d in enumerate((dx, dy, dz)))
        dst = tuple(slice(max(0, d), labels.shape[a] - max(0, -d)) for a, d in enumerate((dx, dy, dz)))
        graph[src] |= (labels[src] == labels[dst]).astype(np.uint32) << np.uint32(bit)
    return np.asfortranarray(graph)
