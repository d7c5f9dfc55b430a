"""Seeded synthetic label volumes with the shapes of the benchmark workloads.

The reference measures on connectomics volumes that are not available here; these generators
stand in for them with the shapes, sizes and object statistics the workloads name:

* ``tube_volume``      random-walk tubes in a box: unit steps, heading turned by a Gaussian angle
                       (sigma 0.2 rad) per step, a branch with probability 0.01 per step, a ball of
                       the tube's radius painted at every step, later ids overwriting earlier ones
                       (the 128^3 uint32 20-object volume, the uneven batch, the serving requests)
* ``dense_volume``     Voronoi cells of uniform seeds intersected with a union of random-walk
                       tubes (one per seed), cell boundaries eroded by one voxel, random 64-bit ids
                       (the 512^3 uint64 and 1024x1024x256 volumes)
* ``uneven_batch``     64 volumes with log-uniform edges in [64, 256]

Every volume is Fortran-ordered (x fastest). Painting and the nearest-seed assignment run with
torch (on the GPU when one is visible); the result does not depend on the device.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = ["tube_volume", "dense_volume", "cell_volume", "uneven_batch", "serving_requests"]

_BALLS: dict = {}


def _device():
    try:
        import torch

        return torch.device("cuda" if torch.cuda.is_available() else "cpu")
    except ImportError:  # pragma: no cover
        return None


def _ball(radius):
    """Integer offsets of the ball of `radius` (rounded to quarter voxels)."""
    key = int(round(radius * 4))
    if key not in _BALLS:
        r = key / 4.0
        n = int(math.ceil(r))
        g = np.arange(-n, n + 1)
        x, y, z = np.meshgrid(g, g, g, indexing="ij")
        inside = x * x + y * y + z * z <= r * r
        _BALLS[key] = np.stack([x[inside], y[inside], z[inside]], axis=1).astype(np.int64)
    return _BALLS[key]


def _walk(rng, shape, start, steps, branch_p, sigma=0.2, limit=None):
    """Centres of a random walk of unit steps (and of its branches) inside `shape`; with `limit`,
    at most that many centres over the walk and all its branches."""
    out = []
    stack = [(tuple(float(c) for c in start), tuple(rng.normal(size=3)), int(steps))]
    hi = [float(s - 1) for s in shape]
    while stack:
        (px, py, pz), (hx, hy, hz), remaining = stack.pop()
        norm = math.sqrt(hx * hx + hy * hy + hz * hz) + 1e-12
        hx, hy, hz = hx / norm, hy / norm, hz / norm
        turns = rng.normal(scale=sigma, size=(remaining, 3)).tolist()
        coins = rng.random(remaining).tolist() if branch_p > 0 else None
        for step in range(remaining):
            tx, ty, tz = turns[step]
            dot = tx * hx + ty * hy + tz * hz
            hx, hy, hz = hx + tx - hx * dot, hy + ty - hy * dot, hz + tz - hz * dot
            norm = math.sqrt(hx * hx + hy * hy + hz * hz) + 1e-12
            hx, hy, hz = hx / norm, hy / norm, hz / norm
            px, py, pz = px + hx, py + hy, pz + hz
            if px < 0 or px > hi[0]:
                hx, px = -hx, min(max(px, 0.0), hi[0])
            if py < 0 or py > hi[1]:
                hy, py = -hy, min(max(py, 0.0), hi[1])
            if pz < 0 or pz > hi[2]:
                hz, pz = -hz, min(max(pz, 0.0), hi[2])
            out.append((px, py, pz))
            if limit is not None and len(out) >= limit:
                return np.asarray(out, np.float64).reshape(-1, 3)
            left = remaining - step - 1
            if coins is not None and coins[step] < branch_p and left > 10:
                stack.append(((px, py, pz), tuple(rng.normal(size=3)), int(left * rng.uniform(0.3, 0.8))))
    return np.asarray(out, np.float64).reshape(-1, 3)


def _paint(volume, centres, radius, value):
    """Paints balls of `radius` at `centres` into the torch volume (flat, Fortran index)."""
    import torch

    if len(centres) == 0:
        return
    shape = volume.shape_f
    c = np.unique(np.rint(centres).astype(np.int64), axis=0)
    off = _ball(radius)
    dev = volume.data.device
    pts = torch.from_numpy(c).to(dev)[:, None, :] + torch.from_numpy(off).to(dev)[None, :, :]
    pts = pts.reshape(-1, 3)
    keep = ((pts >= 0) & (pts < torch.tensor(shape, device=dev))).all(dim=1)
    pts = pts[keep]
    flat = pts[:, 0] + shape[0] * (pts[:, 1] + shape[1] * pts[:, 2])
    volume.data[flat] = value


class _Volume:
    def __init__(self, shape, dtype):
        import torch

        self.shape_f = tuple(int(s) for s in shape)
        self.data = torch.zeros(int(np.prod(self.shape_f)), dtype=dtype, device=_device())

    def numpy(self, dtype):
        arr = self.data.cpu().numpy().astype(dtype, copy=False)
        return np.asfortranarray(arr.reshape(self.shape_f[::-1]).transpose(2, 1, 0))


def tube_volume(shape=(128, 128, 128), objects=20, seed=0, steps=(200, 600), radius=(2.0, 6.0), branch_p=0.01,
                arbor_fraction=0.0, arbor_steps=(5000, 8000), dtype=np.uint32, rng=None):
    """Labels 1..objects, each a random-walk tube; later ids overwrite earlier ones. With
    `arbor_fraction` > 0 that share of the objects are long branched arbors."""
    import torch

    rng = np.random.default_rng(seed) if rng is None else rng
    vol = _Volume(shape, torch.int64)
    for label in range(1, objects + 1):
        arbor = arbor_fraction > 0 and rng.random() < arbor_fraction
        n = int(rng.integers(arbor_steps[0], arbor_steps[1] + 1)) if arbor else int(rng.integers(steps[0], steps[1] + 1))
        start = rng.uniform(0, np.asarray(shape) - 1)
        # an arbor: a trunk of a third of its steps whose branches take the rest
        centres = _walk(rng, shape, start, n // 3, 0.02, limit=n) if arbor else _walk(rng, shape, start, n, branch_p)
        _paint(vol, centres, rng.uniform(*radius), label)
    return vol.numpy(dtype)


def dense_volume(shape=(512, 512, 512), seeds=600, seed=1, radius=(3.0, 10.0), steps=(200, 600), dtype=np.uint64):
    """Voronoi cells of `seeds` uniform seeds intersected with a union of random-walk tubes (one per
    seed), cell boundaries eroded by one voxel, random nonzero unique ids."""
    import torch

    rng = np.random.default_rng(seed)
    shape = tuple(int(s) for s in shape)
    points = rng.uniform(0, np.asarray(shape) - 1, size=(seeds, 3))
    mask = _Volume(shape, torch.uint8)
    for s in range(seeds):
        n = int(rng.integers(steps[0], steps[1] + 1))
        centres = _walk(rng, shape, points[s], n, 0.0)
        _paint(mask, centres, rng.uniform(*radius), 1)
    dev = mask.data.device
    where = torch.nonzero(mask.data, as_tuple=False).squeeze(1)
    sx, sy = shape[0], shape[1]
    coords = torch.stack([where % sx, (where // sx) % sy, where // (sx * sy)], dim=1).to(torch.float64)
    seeds_t = torch.from_numpy(points).to(dev)
    owner = torch.empty(where.numel(), dtype=torch.int64, device=dev)
    chunk = 1 << 20
    for i in range(0, where.numel(), chunk):
        owner[i:i + chunk] = torch.cdist(coords[i:i + chunk], seeds_t).argmin(dim=1)
    cells = torch.zeros(int(np.prod(shape)), dtype=torch.int32, device=dev)
    cells[where] = (owner + 1).to(torch.int32)
    c3 = cells.view(shape[2], shape[1], shape[0])  # (z, y, x)
    boundary = torch.zeros_like(c3, dtype=torch.bool)
    for axis in range(3):
        a = [slice(None)] * 3
        b = [slice(None)] * 3
        a[axis], b[axis] = slice(1, None), slice(None, -1)
        u, v = c3[tuple(a)], c3[tuple(b)]
        diff = (u != v) & (u != 0) & (v != 0)
        boundary[tuple(a)] |= diff
        boundary[tuple(b)] |= diff
    c3[boundary] = 0
    info = np.iinfo(dtype)
    draw = rng.integers(1, min(int(info.max), 2 ** 63 - 1), size=seeds * 2, dtype=np.int64).astype(dtype)
    ids = np.unique(draw)
    ids = ids[ids != 0]
    rng.shuffle(ids)
    lut = np.zeros(seeds + 1, dtype=dtype)
    lut[1:] = ids[:seeds]
    cells_np = c3.cpu().numpy()  # (z, y, x) C order == Fortran (x, y, z)
    return np.asfortranarray(lut[cells_np].transpose(2, 1, 0))


def cell_volume(shape=(256, 256, 256), cells=64, seed=6, nucleus=(0.35, 0.5), cavity_share=0.5, dtype=np.uint32):
    """Voronoi cells of `cells` uniform seeds filling the volume (boundaries eroded by one voxel),
    each with a nucleus: a ball of its own label around the seed, of a radius that is a fraction
    (`nucleus`) of the seed's distance to its nearest other seed; about `cavity_share` of the cells
    also hold an empty cavity beside the nucleus. The nuclei are the pits the avocado stage merges
    into their cells, the cavities the voids hole filling fills. Labels: cells 1..cells, nuclei
    cells+1..2*cells."""
    import torch

    rng = np.random.default_rng(seed)
    shape = tuple(int(s) for s in shape)
    dev = _device()
    points = rng.uniform(4, np.asarray(shape) - 5, size=(cells, 3))
    seeds_t = torch.from_numpy(points).to(dev)
    n = int(np.prod(shape))
    sx, sy = shape[0], shape[1]
    owner = torch.empty(n, dtype=torch.int64, device=dev)
    near = torch.empty(n, dtype=torch.float64, device=dev)
    chunk = 1 << 20
    for i in range(0, n, chunk):
        idx = torch.arange(i, min(n, i + chunk), device=dev)
        coords = torch.stack([idx % sx, (idx // sx) % sy, idx // (sx * sy)], dim=1).to(torch.float64)
        d = torch.cdist(coords, seeds_t)
        near[i:i + chunk], owner[i:i + chunk] = d.min(dim=1)
    labels = (owner + 1).to(torch.int64)
    spacing = torch.cdist(seeds_t, seeds_t) + torch.eye(cells, device=dev, dtype=torch.float64) * 1e9
    gap = spacing.min(dim=1).values  # each seed's distance to its nearest other seed
    frac = torch.from_numpy(rng.uniform(*nucleus, size=cells)).to(dev)
    radius = gap * frac / 2
    inside = near <= radius[owner]
    labels[inside] = owner[inside] + 1 + cells
    # a cavity: a ball of half the nucleus's radius centred beside it, in half of the cells
    with_cavity = torch.from_numpy(rng.random(cells) < cavity_share).to(dev)
    direction = torch.from_numpy(rng.normal(size=(cells, 3))).to(dev)
    direction = direction / direction.norm(dim=1, keepdim=True)
    centre = seeds_t + direction * (radius * 1.9)[:, None]
    for i in range(0, n, chunk):
        idx = torch.arange(i, min(n, i + chunk), device=dev)
        o = owner[i:i + chunk]
        coords = torch.stack([idx % sx, (idx // sx) % sy, idx // (sx * sy)], dim=1).to(torch.float64)
        dc = (coords - centre[o]).norm(dim=1)
        hole = with_cavity[o] & (dc <= radius[o] * 0.5) & ~inside[i:i + chunk]
        labels[i:i + chunk][hole] = 0
    c3 = labels.view(shape[2], shape[1], shape[0])
    boundary = torch.zeros_like(c3, dtype=torch.bool)
    for axis in range(3):
        a = [slice(None)] * 3
        b = [slice(None)] * 3
        a[axis], b[axis] = slice(1, None), slice(None, -1)
        u, v = c3[tuple(a)], c3[tuple(b)]
        cell_u, cell_v = (u - 1) % cells, (v - 1) % cells  # a nucleus and its cell stay joined
        diff = (u != 0) & (v != 0) & (cell_u != cell_v)
        boundary[tuple(a)] |= diff
        boundary[tuple(b)] |= diff
    c3[boundary] = 0
    return np.asfortranarray(c3.cpu().numpy().astype(dtype).transpose(2, 1, 0))


def uneven_batch(count=64, seed=2, edges=(64, 256), tubes=(10, 80), radius=(1.0, 8.0), arbor_fraction=0.05):
    """`count` uint32 volumes, each axis log-uniform in `edges`, filled with tubes (about 5% of the
    objects are long branched arbors)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        shape = tuple(int(round(math.exp(rng.uniform(math.log(edges[0]), math.log(edges[1]))))) for _ in range(3))
        out.append(tube_volume(shape, int(rng.integers(tubes[0], tubes[1] + 1)), rng=rng, radius=radius,
                               arbor_fraction=arbor_fraction))
    return out


def serving_requests(count, rate, seed=4, edges=(32, 384)):
    """Poisson arrivals at `rate` per second: (arrival time, volume) with log-uniform edges, one tube
    per 64^3 voxels, uint32 or uint64 with equal probability."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=count))
    out = []
    for i in range(count):
        shape = tuple(int(round(math.exp(rng.uniform(math.log(edges[0]), math.log(edges[1]))))) for _ in range(3))
        tubes = max(1, int(round(np.prod(shape) / 64 ** 3)))
        dtype = np.uint32 if rng.random() < 0.5 else np.uint64
        out.append((float(t[i]), tube_volume(shape, tubes, rng=rng, dtype=dtype)))
    return out
