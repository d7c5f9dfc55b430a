"""Seeded packed skeleton sets for the post-processing tests: per label a few components, each a
random tree on a random walk of vertices (integer-valued coordinates, so distances tie), with
extra edges that close cycles of every kind (no branch node, one, two, three or more), short
terminal branches, near components that join and far ones that do not, isolated vertices and
empty labels."""
from __future__ import annotations

import numpy as np


def _component(rng, start, size, spacing):
    pts = [np.asarray(start, np.float64)]
    parent = [-1]
    for i in range(1, size):
        p = int(rng.integers(0, i)) if rng.random() < 0.35 else i - 1
        step = rng.integers(-1, 2, 3) * spacing
        if not step.any():
            step[0] = spacing[0]
        pts.append(pts[p] + step)
        parent.append(p)
    edges = [(parent[i], i) for i in range(1, size)]
    return np.asarray(pts), edges


def packed_set(seed, labels=6, max_components=4, max_size=60, cycles=3, spacing=(8.0, 8.0, 40.0), oriented=True):
    rng = np.random.default_rng(seed)
    spacing = np.asarray(spacing)
    out = dict(labels=[], vertex_offsets=[0], edge_offsets=[0], vertices=[], edges=[], radii=[])
    for l in range(labels):
        verts, edges = [], []
        if rng.random() < 0.1:  # an empty label
            out["labels"].append(1000 + l)
            out["vertex_offsets"].append(out["vertex_offsets"][-1])
            out["edge_offsets"].append(out["edge_offsets"][-1])
            continue
        origin = rng.integers(0, 50, 3) * spacing
        for c in range(int(rng.integers(1, max_components + 1))):
            size = int(rng.integers(1, max_size))
            # near (joinable) or far from the previous component
            shift = rng.integers(-3, 4, 3) * spacing if rng.random() < 0.6 else rng.integers(30, 60, 3) * spacing
            pts, es = _component(rng, origin + shift * c, size, spacing)
            base = len(verts)
            verts.extend(pts.tolist())
            edges.extend((a + base, b + base) for a, b in es)
            for _ in range(int(rng.integers(0, cycles + 1))):
                if size > 3:
                    a, b = rng.choice(size, 2, replace=False)
                    if (a + base, b + base) not in edges and (b + base, a + base) not in edges:
                        edges.append((int(a) + base, int(b) + base))
        if rng.random() < 0.2:  # an isolated vertex
            verts.append((origin + rng.integers(0, 5, 3) * spacing).tolist())
        order = rng.permutation(len(edges))
        edges = [edges[i] for i in order]
        if not oriented:
            edges = [(b, a) if rng.random() < 0.5 else (a, b) for a, b in edges]
        else:
            edges = [(min(a, b), max(a, b)) for a, b in edges]
        out["labels"].append(1000 + l)
        out["vertex_offsets"].append(out["vertex_offsets"][-1] + len(verts))
        out["edge_offsets"].append(out["edge_offsets"][-1] + len(edges))
        out["vertices"].extend(verts)
        out["edges"].extend(edges)
        out["radii"].extend((rng.integers(1, 12, len(verts)) * 4.0).tolist())
    return dict(labels=np.asarray(out["labels"], np.int64),
                vertex_offsets=np.asarray(out["vertex_offsets"], np.int64),
                edge_offsets=np.asarray(out["edge_offsets"], np.int64),
                vertices=np.asarray(out["vertices"], np.float32).reshape(-1, 3),
                edges=np.asarray(out["edges"], np.uint32).reshape(-1, 2),
                radii=np.asarray(out["radii"], np.float32))


def to_packed(d, anisotropy=(8.0, 8.0, 40.0)):
    from brook_b200 import PackedSkeletons

    return PackedSkeletons(d["labels"], d["vertex_offsets"], d["edge_offsets"], d["vertices"], d["edges"], d["radii"],
                           tuple(anisotropy))


def from_packed(p):
    h = p.to_host()
    return dict(labels=np.asarray(h.labels), vertex_offsets=np.asarray(h.v_off), edge_offsets=np.asarray(h.e_off),
                vertices=np.asarray(h.vertices).reshape(-1, 3), edges=np.asarray(h.edges).reshape(-1, 2),
                radii=np.asarray(h.radii))


def assert_same_packed(got, exp, what=""):
    for key in ("labels", "vertex_offsets", "edge_offsets", "edges"):
        np.testing.assert_array_equal(np.asarray(got[key]), np.asarray(exp[key]), err_msg=f"{what} {key}")
    for key in ("vertices", "radii"):
        np.testing.assert_array_equal(np.asarray(got[key]).view(np.uint32), np.asarray(exp[key]).view(np.uint32),
                                      err_msg=f"{what} {key} bits")
