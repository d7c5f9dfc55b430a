"""Synthetic label volumes of the reference's join tests and the digest its expectations use.

The shapes and the expected summaries are the reference's own known answers
(tests/python/test_package.py:2019-2113 of giorgioangel/brook: Kimimaro 5.8.1 with dijkstra3d
1.15.2 under the options `JOIN_OPTIONS`); `make_golden.py` writes them to `join_digests.json`.
The generators here compute the same volumes from the same formulas.
"""
from __future__ import annotations

import hashlib

import numpy as np

JOIN_OPTIONS = dict(teasar_params=dict(scale=1.0, const=2.0), anisotropy=(4, 4, 4), dust_threshold=0,
                    fix_branching=True, fix_borders=True)


def sine_band(amplitude, period, width, phase=0.0, axis=0):
    """|y - (32 + amplitude sin(2 pi x / period + phase))| < width on a 64 x 160 plane, one voxel
    thick along `axis`."""
    y, x = np.mgrid[:64, :160]
    band = np.abs(y - (32 + amplitude * np.sin(2 * np.pi * x / period + phase))) < width
    return np.moveaxis(band[None].astype(np.uint32), 0, axis)


def sine_bands():
    """Labels 1..3 as three bands of one 64 x 160 plane, each painted where the earlier ones left 0."""
    y, x = np.mgrid[:64, :160]
    plane = np.zeros((64, 160), np.uint32)
    for label, (centre, amplitude, period, width) in enumerate([(12, 4, 50, 1.7), (30, 6, 70, 2.2), (48, 5, 45, 1.5)], 1):
        plane[(np.abs(y - (centre + amplitude * np.sin(2 * np.pi * x / period))) < width) & (plane == 0)] = label
    return plane[None]


def spiral_band():
    """A one-voxel-thick spiral band in a 96 x 96 plane, turns 11 voxels apart."""
    y, x = np.mgrid[:96, :96]
    r, angle = np.hypot(y - 47.3, x - 48.6), np.mod(np.arctan2(y - 47.3, x - 48.6), 2 * np.pi)
    turn = (r - 6 - 5.5 * angle / np.pi) / 11.0
    return ((np.abs(turn - np.round(turn)) * 11.0 < 1.8) & (r > 5) & (r < 44))[None].astype(np.uint32)


def helix_tube(radius, turn_radius, pitch, length):
    """A tube of the given radius around a helix along x."""
    n = int(2 * turn_radius + 2 * radius + 6)
    x = np.arange(length, dtype=np.float64)[:, None, None]
    y = np.arange(n, dtype=np.float64)[None, :, None]
    z = np.arange(n, dtype=np.float64)[None, None, :]
    cy, cz = n / 2 + turn_radius * np.cos(2 * np.pi * x / pitch), n / 2 + turn_radius * np.sin(2 * np.pi * x / pitch)
    return ((y - cy) ** 2 + (z - cz) ** 2 <= radius * radius).astype(np.uint32)


CASES = {
    "band_axis0": (lambda: sine_band(6.0, 60.0, 1.6, axis=0), {}),
    "band_axis1": (lambda: sine_band(6.0, 60.0, 1.6, axis=1), {}),
    "band_axis2": (lambda: sine_band(6.0, 60.0, 1.6, axis=2), {}),
    "bands": (sine_bands, {}),
    "wide": (lambda: sine_band(9.0, 80.0, 2.1, 0.7), {}),
    "spiral": (spiral_band, {"anisotropy": (1, 1, 1)}),
    "helix": (lambda: helix_tube(1.9, 8.0, 28.0, 28), {}),
}


def digest(vertices, edges, radii):
    """Order-independent exact digest of one skeleton: its (vertex, radius) rows and its edges."""
    rows = np.column_stack([np.asarray(vertices), np.asarray(radii)]).astype(np.float32)
    order = np.lexsort(rows.T[::-1])
    rank = np.empty(len(order), np.int64)
    rank[order] = np.arange(len(order))
    e = np.sort(rank[np.asarray(edges, np.int64)], axis=1).reshape(-1, 2)
    e = e[np.lexsort(e.T[::-1])]
    return hashlib.sha256(rows[order].tobytes() + e.tobytes()).hexdigest()[:16]


def summary(skeletons):
    """{label: [vertices, edges, largest radius, digest]} of {label: (vertices, edges, radii)}."""
    return {int(label): [len(v), len(e), float(np.max(r)), digest(v, e, r)] for label, (v, e, r) in skeletons.items()}
