"""CPU restatement of the merge of skeleton fragments (the reference's merge_parts and
merge_fragments, cpp/src/packed_merge.cu:88-166 and cpp/src/packed.cpp:67-86, with its defaults:
labels sorted ascending, labels without edges kept).

TEST INFRASTRUCTURE ONLY: the checker of brook_b200's device merge; the product never imports it.

Each fragment is a dict of packed arrays (labels, vertex_offsets, edge_offsets, vertices (V, 3),
edges (E, 2), radii) and an origin (physical units) added to its vertices in float32. Vertices of
one label at the same point merge (float32 equality, -0 == +0, NaN never equal), keeping the
radius of their first occurrence in fragment order; edges map onto the merged vertices, self loops
drop, duplicates collapse; vertices on no edge drop; per label, vertices sorted by (x, y, z) with
NaN last, edges as sorted (lower, higher) local pairs.
"""
from __future__ import annotations

import numpy as np


def merge(fragments, origins):
    labels = sorted({int(l) for f in fragments for k, l in enumerate(f["labels"])
                     if f["vertex_offsets"][k + 1] > f["vertex_offsets"][k]})
    group_of = {l: g for g, l in enumerate(labels)}
    coords, radii, groups, edges = [], [], [], []
    base = 0
    for f, origin in zip(fragments, origins):
        o = np.asarray(origin, np.float32)
        for k, l in enumerate(f["labels"]):
            v0, v1 = int(f["vertex_offsets"][k]), int(f["vertex_offsets"][k + 1])
            e0, e1 = int(f["edge_offsets"][k]), int(f["edge_offsets"][k + 1])
            if v1 == v0:
                continue
            coords.append(np.asarray(f["vertices"][v0:v1], np.float32) + o)
            radii.append(np.asarray(f["radii"][v0:v1], np.float32))
            groups.append(np.full(v1 - v0, group_of[int(l)], np.int64))
            edges.append(np.asarray(f["edges"][e0:e1], np.int64).reshape(-1, 2) + base)
            base += v1 - v0
    out = dict(labels=np.asarray(labels, np.int64), vertex_offsets=np.zeros(len(labels) + 1, np.int64),
               edge_offsets=np.zeros(len(labels) + 1, np.int64), vertices=np.zeros((0, 3), np.float32),
               edges=np.zeros((0, 2), np.uint32), radii=np.zeros(0, np.float32))
    if not coords:
        return out
    xyz = np.concatenate(coords) + np.float32(0)  # -0 -> +0
    rad, grp = np.concatenate(radii), np.concatenate(groups)
    order = np.lexsort((xyz[:, 2], xyz[:, 1], xyz[:, 0], grp))  # stable; NaN sorts last
    s = xyz[order]
    new = np.ones(len(order), bool)
    new[1:] = (grp[order][1:] != grp[order][:-1]) | np.any(s[1:] != s[:-1], axis=1)
    rank = np.cumsum(new) - 1
    merged = np.empty(len(order), np.int64)
    merged[order] = rank
    first = order[new]
    e = np.concatenate(edges) if edges else np.zeros((0, 2), np.int64)
    a, b = merged[e[:, 0]], merged[e[:, 1]]
    keep = a != b
    pairs = np.unique(np.stack([np.minimum(a, b)[keep], np.maximum(a, b)[keep]], axis=1), axis=0)
    used = np.zeros(len(first), bool)
    used[pairs.ravel()] = True
    new_id = np.cumsum(used) - 1
    vgroup = grp[first]
    vcount = np.bincount(vgroup[used], minlength=len(labels))
    ecount = np.bincount(vgroup[pairs[:, 0]], minlength=len(labels)) if len(pairs) else np.zeros(len(labels), np.int64)
    out["vertex_offsets"] = np.concatenate([[0], np.cumsum(vcount)]).astype(np.int64)
    out["edge_offsets"] = np.concatenate([[0], np.cumsum(ecount)]).astype(np.int64)
    out["vertices"] = xyz[first[used]]
    out["radii"] = rad[first[used]]
    local = new_id[pairs] - out["vertex_offsets"][vgroup[pairs[:, 0]]][:, None]
    out["edges"] = local.astype(np.uint32).reshape(-1, 2)
    return out
