"""Float64 shortest-path distances over a component's 26-connected voxel graph, for checking the
float32 distance fields (the DAF floods and the railroad searches) against exact arithmetic.

The float32 fields sum their steps in float32, as the reference does; a path of h steps carries at
most h roundings of half an ulp each, plus, in the railroad, a one-ulp advance where a step is
absorbed (vw_step). So a float32 distance is within (h + 2) * 2**-23 relative of the float64
distance, h being the float64 path's step count; `hops` gives h per voxel."""
import numpy as np
from scipy.sparse import csr_matrix
from scipy.sparse.csgraph import dijkstra

OFFSETS = [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if dx or dy or dz]
ULP_BOUND = 2.0 ** -23


def neighbour_graph(mask, weight):
    """(voxel flat indices (F order), flat -> vertex map, CSR graph): an edge u -> v for every pair
    of 26-neighbours in `mask`, weighted weight(dx, dy, dz, v_flat) (float64 arrays)."""
    sx, sy, sz = mask.shape
    flat_mask = mask.ravel(order="F")
    idx = np.flatnonzero(flat_mask)
    pos = np.full(mask.size, -1, np.int64)
    pos[idx] = np.arange(idx.size)
    x, y, z = idx % sx, (idx // sx) % sy, idx // (sx * sy)
    rows, cols, vals = [], [], []
    for dx, dy, dz in OFFSETS:
        nx, ny, nz = x + dx, y + dy, z + dz
        ok = (nx >= 0) & (nx < sx) & (ny >= 0) & (ny < sy) & (nz >= 0) & (nz < sz)
        f = np.where(ok, nx + sx * (ny + sy * nz), 0)
        ok &= flat_mask[f]
        rows.append(np.flatnonzero(ok))
        cols.append(pos[f[ok]])
        vals.append(np.asarray(weight(dx, dy, dz, f[ok]), np.float64))
    g = csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(idx.size, idx.size))
    return idx, pos, g


def hops(pred):
    """Steps from the source along a scipy predecessor tree (-9999 at the source and unreached)."""
    depth = (pred >= 0).astype(np.int64)
    anc = np.where(pred >= 0, pred, -1)
    while (anc >= 0).any():
        ok = anc >= 0
        nd, na = depth.copy(), anc.copy()
        nd[ok] += depth[anc[ok]]
        na[ok] = anc[anc[ok]]
        depth, anc = nd, na
    return depth


def geometric_distances(mask, source, anisotropy):
    """Float64 distances from flat voxel `source` over `mask`, a step costing the distance between
    the voxel centres; returns (voxel flat indices, distances, hops)."""
    a = np.asarray(anisotropy, np.float64)
    idx, pos, g = neighbour_graph(mask, lambda dx, dy, dz, v: np.full(v.size, np.sqrt(
        (dx * a[0]) ** 2 + (dy * a[1]) ** 2 + (dz * a[2]) ** 2)))
    d, pred = dijkstra(g, indices=pos[source], return_predecessors=True)
    return idx, d, hops(pred)


def vertex_weighted_distances(mask, source, field):
    """Float64 distances from flat voxel `source` over `mask`, entering voxel v costing field[v]
    (all positive on `mask`); returns (voxel flat indices, distances, hops)."""
    flat = np.asarray(field, np.float32).ravel(order="F").astype(np.float64)
    idx, pos, g = neighbour_graph(mask, lambda dx, dy, dz, v: flat[v])
    d, pred = dijkstra(g, indices=pos[source], return_predecessors=True)
    return idx, d, hops(pred)


def relative_errors(got, exact):
    """|got - exact| / exact, 0 where both are 0."""
    got = np.asarray(got, np.float64)
    rel = np.abs(got - exact) / np.where(exact > 0, exact, 1.0)
    rel[(exact == 0) & (got == 0)] = 0.0
    return rel
