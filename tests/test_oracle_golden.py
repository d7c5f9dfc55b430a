"""The CPU oracle against the reference's own known answers (CPU only)."""
import itertools
import json
import os

import numpy as np
import pytest

import shapes
from oracle import oracle

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "join_digests.json")))


@pytest.mark.parametrize("case", sorted(shapes.CASES))
@pytest.mark.parametrize("layout", [np.ascontiguousarray, np.asfortranarray])
def test_join_digests(case, layout):
    """Kimimaro 5.8.1 + dijkstra3d 1.15.2 summaries the reference pins (test_package.py:2079-2113)."""
    make, extra = shapes.CASES[case]
    result = oracle.skeletonize(layout(make()), **dict(shapes.JOIN_OPTIONS, **extra))
    assert shapes.summary(result.skeletons()) == {int(k): v for k, v in GOLDEN[case].items()}


def _flat(p, shape):
    return int(np.ravel_multi_index(p, shape, order="F"))


def test_railroad_plane_and_wall():
    """test_package.py:751-778: the lowest-flat nearest rail fixes the last road voxel, and the
    path joins that voxel's first rail in dijkstra3d order; a walled target has no path."""
    field = np.ones((9, 9, 9), np.float32, order="F")
    field[:, :, 0] = 0
    target = _flat((4, 4, 4), field.shape)
    road = [(4, 4, 4), (3, 3, 3), (2, 2, 2), (1, 1, 1), (1, 1, 0)]
    assert oracle.railroad(field, target) == [_flat(p, field.shape) for p in road]
    walled = field.copy(order="F")
    walled[2:7, 2:7, 2:7] = np.inf
    walled[3:6, 3:6, 3:6] = 1
    assert oracle.railroad(walled, target) == []


D3_ORDER = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1),
            (-1, -1, 0), (-1, 1, 0), (1, -1, 0), (1, 1, 0), (0, -1, -1), (0, -1, 1), (0, 1, -1), (0, 1, 1),
            (-1, 0, -1), (-1, 0, 1), (1, 0, -1), (1, 0, 1),
            (-1, -1, -1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1), (1, 1, -1), (1, -1, 1), (-1, 1, 1), (1, 1, 1)]


def test_railroad_join_order():
    """test_package.py:782-811: every single rail, every pair and all 26 around the target: the
    path joins the first rail in dijkstra3d's neighbour order."""
    shape, centre = (5, 5, 5), (2, 2, 2)
    near = [tuple(c + d for c, d in zip(centre, o)) for o in D3_ORDER]
    for rails in [(i,) for i in range(26)] + list(itertools.combinations(range(26), 2)) + [tuple(range(26))]:
        field = np.ones(shape, np.float32, order="F")
        for i in rails:
            field[near[i]] = 0
        assert oracle.railroad(field, _flat(centre, shape)) == [_flat(centre, shape), _flat(near[rails[0]], shape)], rails


def test_railroad_join_order_with_voxel_graph():
    """test_package.py:802-808: for every pair of rails, the first one's direction cut from the
    voxel graph at the target: the path joins the second (dijkstra3d 1.15.2's answers)."""
    from oracle import graph as og

    shape, centre = (5, 5, 5), (2, 2, 2)
    near = [tuple(c + d for c, d in zip(centre, o)) for o in D3_ORDER]
    for rails in itertools.combinations(range(26), 2):
        field = np.ones(shape, np.float32, order="F")
        for i in rails:
            field[near[i]] = 0
        graph = np.full(shape, (1 << 26) - 1, np.uint32, order="F")
        graph[centre] &= ~np.uint32(1 << og.STEPS.index(D3_ORDER[rails[0]]))
        path = oracle.railroad(field, _flat(centre, shape), voxel_graph=graph)
        assert path == [_flat(centre, shape), _flat(near[rails[1]], shape)], rails
    # an all-permitting graph changes nothing; a graph that permits no step leaves no path
    field = np.ones(shape, np.float32, order="F")
    field[near[5]] = 0
    assert oracle.railroad(field, _flat(centre, shape), voxel_graph=np.full(shape, (1 << 26) - 1, np.uint32)) == \
        oracle.railroad(field, _flat(centre, shape))
    assert oracle.railroad(field, _flat(centre, shape), voxel_graph=np.zeros(shape, np.uint32)) == []


def test_edt_line():
    """c_smoke.c:45-61: EDT of an 8-voxel line {1,1,0,0,0,0,2,2}, anisotropy 1, no black border."""
    labels = np.array([1, 1, 0, 0, 0, 0, 2, 2], np.uint32).reshape(8, 1, 1)
    d = oracle.edt(labels, (1, 1, 1), False).ravel()
    assert d[0] == 2 and d[1] == 1 and d[2] == 0 and d[6] == 1 and d[7] == 2


def test_target_order_rule():
    """component_order_smoke.cpp:10-29: descending DAF, infinity and -0 as 0, ties -> higher index,
    on the reference's own generator (std::mt19937(482))."""
    bits = np.random.MT19937(0)
    bits._legacy_seeding(482)
    raw = lambda: int(bits.random_raw())
    for n in (1, 17, 1025):
        for density in (0, 3, 50, 100):
            for ties in (1, 7, 10000):
                mask = np.zeros(n, np.uint8)
                daf = np.zeros(n, np.float32)
                for i in range(n):
                    mask[i] = (1 + raw() % 7) if raw() % 100 < density else 0
                    daf[i] = np.float32(raw() % ties) * np.float32(0.37)
                    if i % 19 == 0:
                        daf[i] = np.inf
                    if i % 23 == 0:
                        daf[i] = -0.0
                got = oracle.target_order(mask, daf)
                key = np.where(np.isinf(daf), 0, daf).astype(np.float64)
                idx = np.nonzero(mask)[0]
                expected = sorted(idx.tolist(), key=lambda i: (-key[i], -i))
                assert got.tolist() == expected


def _scipy_edt(labels, anisotropy, black_border):
    """The multi-label EDT in float64: per label, the exact Euclidean distance transform of its
    voxels (distance to the nearest voxel of another label or background); with black border the
    volume is padded by background first."""
    from scipy import ndimage

    pad = 1 if black_border else 0
    lab = np.pad(labels, pad) if pad else labels
    out = np.zeros(lab.shape, np.float64)
    for value in np.unique(lab):
        if value == 0:
            continue
        inside = lab == value
        if inside.all():  # no other voxel anywhere: the distance is unbounded
            out[inside] = np.inf
            continue
        out[inside] = ndimage.distance_transform_edt(inside, sampling=anisotropy)[inside]
    return out[pad:lab.shape[0] - pad, pad:lab.shape[1] - pad, pad:lab.shape[2] - pad] if pad else out


def test_edt_within_1e6_of_float64():
    """The float32 EDT (float32 spacing table, float64 envelope) within 1e-6 relative of an exact
    float64 transform, on multi-label volumes, anisotropic spacings and with black border."""
    from scipy import ndimage

    rng = np.random.default_rng(11)
    for shape, aniso, bb in (((30, 24, 18), (1, 1, 1), False), ((26, 20, 22), (8, 8, 40), True),
                             ((20, 28, 16), (7.91, 7.91, 7.91), False), ((40, 12, 10), (4, 5, 6), True)):
        field = ndimage.gaussian_filter(rng.random((4,) + shape), sigma=(0, 2, 2, 2))
        labels = np.asfortranarray((np.argmax(field, axis=0) + 1).astype(np.uint32))
        labels[rng.random(shape) < 0.05] = 0
        got = oracle.edt(labels, aniso, bb).astype(np.float64)
        exp = _scipy_edt(labels, aniso, bb)
        finite = np.isfinite(exp)
        assert np.array_equal(np.isfinite(got), finite)
        rel = np.abs(got[finite] - exp[finite]) / np.maximum(exp[finite], 1e-30)
        assert rel.max() <= 1e-6, (shape, aniso, bb, rel.max())


@pytest.mark.parametrize("fix_branching", [True, False])
def test_oracle_answers_that_follow_from_teasar_alone(fix_branching):
    """Answers that hold for any TEASAR with the reference's object rules, with and without
    fix_branching: a one-voxel-thick line is its own skeleton; an object whose bounding box is one
    voxel, or whose voxel count is within the dust threshold, has none (batched.cu:187-191)."""
    line = np.zeros((30, 3, 3), np.uint32)
    line[3:27, 1, 1] = 7
    p = oracle.skeletonize(line, anisotropy=(4, 5, 6), dust_threshold=0, fix_branching=fix_branching).packed()
    assert p["labels"].tolist() == [7]
    verts = p["vertices"].reshape(-1, 3)
    assert len(verts) == 24 and len(p["edges"].reshape(-1, 2)) == 23
    assert sorted(verts[:, 0].tolist()) == [4.0 * x for x in range(3, 27)]
    assert set(verts[:, 1].tolist()) == {5.0} and set(verts[:, 2].tolist()) == {6.0}
    edges = {tuple(sorted(e)) for e in p["edges"].reshape(-1, 2).tolist()}
    order = np.argsort(verts[:, 0])
    assert edges == {tuple(sorted((int(order[i]), int(order[i + 1])))) for i in range(23)}

    dots = np.zeros((10, 10, 10), np.uint32)
    dots[2, 2, 2] = 1                 # one voxel: no skeleton
    dots[6, 6, 6] = dots[6, 6, 7] = 2  # two voxels: one edge
    dots[0:4, 8, 8] = 3               # four voxels
    p = oracle.skeletonize(dots, anisotropy=(1, 1, 1), dust_threshold=0, fix_branching=fix_branching).packed()
    assert p["labels"].tolist() == [2, 3]
    p = oracle.skeletonize(dots, anisotropy=(1, 1, 1), dust_threshold=3, fix_branching=fix_branching).packed()
    assert p["labels"].tolist() == [3]  # 2 voxels <= dust 3 < 4
    assert oracle.skeletonize(np.zeros((5, 5, 5), np.uint8), dust_threshold=0).packed()["labels"].size == 0


def test_branching_off_y_shape_keeps_every_branch_to_the_root():
    """Without fix_branching every path runs back to the root through one shortest-path tree
    (trace.cu:151-160): on a one-voxel-thick Y the skeleton is the Y itself, one connected tree."""
    y = np.zeros((40, 40, 3), np.uint32)
    for i in range(18):
        y[20, 2 + i, 1] = 1          # the stem
        y[20 - i, 20 + i, 1] = 1     # one arm
        y[20 + i, 20 + i, 1] = 1     # the other
    p = oracle.skeletonize(y, teasar_params=dict(scale=1, const=1), anisotropy=(1, 1, 1), dust_threshold=0,
                           fix_branching=False, fix_borders=False).packed()
    verts = p["vertices"].reshape(-1, 3)
    assert len(verts) == int((y > 0).sum())
    assert len(p["edges"].reshape(-1, 2)) == len(verts) - 1  # a tree over every voxel


def test_oracle_threads_and_steps_do_not_change_the_result():
    """The oracle's threaded preamble (slab-wise components, line-parallel EDT, per-object floods
    and orders) and its stepped form (oracle.StagedRun: the trace split over sub-ranges of the
    object order) give the single-threaded one-shot result exactly."""
    from brook_b200 import synthetic

    labels = synthetic.dense_volume((80, 72, 64), seeds=30, seed=11, dtype=np.uint32)
    opts = dict(teasar_params=dict(scale=1.5, const=300, pdrf_scale=100000, pdrf_exponent=4), anisotropy=(8, 8, 40),
                dust_threshold=50)
    one = oracle.skeletonize(labels, threads=1, stages=True, **opts)
    many = oracle.skeletonize(labels, threads=6, stages=True, **opts)
    for name in ("cc", "dbf", "daf", "pdrf", "roots", "targets", "orders", "labels", "vertices", "edges", "radii"):
        np.testing.assert_array_equal(one.array(name), many.array(name), err_msg=name)
    run = oracle.StagedRun(labels, threads=3, **opts)
    assert run.objects > 10
    for b in range(0, run.objects, 7):
        run.trace(b, b + 7)
    stepped = run.finish().packed()
    for name, value in one.packed().items():
        np.testing.assert_array_equal(stepped[name], value, err_msg=name)


def _soma_with_processes(size=72, centre=36, radius=12):
    """The reference's soma test shape (test_package.py:343-366): a ball with a three-voxel-thick
    process along each axis through its centre."""
    grid = np.indices((size,) * 3) - centre
    labels = ((grid ** 2).sum(axis=0) <= radius ** 2).astype(np.uint8)
    for axis in range(3):
        tube = [slice(centre - 1, centre + 2)] * 3
        tube[axis] = slice(2, size - 2)
        labels[tuple(tube)] = 1
    return np.asfortranarray(labels)


SOMA_PARAMS = dict(scale=1.5, const=2, pdrf_scale=100000, pdrf_exponent=4, soma_detection_threshold=6,
                   soma_acceptance_threshold=9, soma_invalidation_scale=1.0, soma_invalidation_const=2)


def _components(vertices, edges):
    parent = list(range(len(vertices)))

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for a, b in edges:
        parent[find(a)] = find(b)
    return len({find(i) for i in range(len(vertices))})


@pytest.mark.parametrize("fix_branching", [True, False])
@pytest.mark.parametrize("hollow", [False, True])
def test_soma_paths_stay_attached(fix_branching, hollow):
    """The reference's soma known answers (test_package.py:343-366), with and without
    fix_branching: every process is traced, the soma root (the centre) is a vertex, and the
    skeleton is one connected tree. `hollow` adds a cavity inside the soma: the filled crop's
    recomputed DBF gives the same answers."""
    labels = _soma_with_processes()
    if hollow:
        labels[33:40, 30:34, 33:40] = 0  # a void the processes do not cross, filled before tracing
    verts, edges, _ = oracle.skeletonize(labels, teasar_params=SOMA_PARAMS, dust_threshold=0,
                                         fix_branching=fix_branching, fix_borders=False).skeletons()[1]
    offsets = np.abs(verts - 36)
    assert (offsets.max(axis=1) > 30).sum() >= 6, "every process is traced"
    assert np.any(np.all(verts == 36, axis=1)), "the soma root is a vertex"
    assert _components(verts, edges) == 1
    # no path vertex well inside the soma radius (about the ball's radius + 2) but the root: the
    # paths are trimmed to it
    inside = np.sqrt((offsets ** 2).sum(axis=1)) <= 10
    assert inside.sum() == 1


def test_merge_restatement_joins_overlapping_chunks_of_a_line():
    """The merge of fragments (oracle/merge.py): a one-voxel line cut into two chunks overlapping
    by one voxel merges back into the whole line's skeleton, and a label seen in one chunk only
    passes through."""
    from oracle import merge as om

    line = np.zeros((40, 3, 3), np.uint32)
    line[2:38, 1, 1] = 5
    line[30:33, 0, 0] = 9
    aniso = (4, 5, 6)
    opts = dict(teasar_params=dict(scale=1, const=1), anisotropy=aniso, dust_threshold=0, fix_borders=True)
    whole = oracle.skeletonize(line, **opts).packed()
    parts = [oracle.skeletonize(np.asfortranarray(line[:21]), **opts).packed(),
             oracle.skeletonize(np.asfortranarray(line[20:]), **opts).packed()]
    merged = om.merge(parts, [(0, 0, 0), (20 * 4, 0, 0)])
    assert merged["labels"].tolist() == [5, 9]  # ascending (the whole volume lists 9 first)

    def per_label(p):
        out = {}
        for k, l in enumerate(p["labels"].tolist()):
            v0, v1, e0, e1 = p["vertex_offsets"][k], p["vertex_offsets"][k + 1], p["edge_offsets"][k], p["edge_offsets"][k + 1]
            out[l] = (p["vertices"].reshape(-1, 3)[v0:v1], p["edges"].reshape(-1, 2)[e0:e1])
        return out

    got, exp = per_label(merged), per_label(whole)
    for l in (5, 9):  # vertices and edges; radii are the chunks' own DBF, which differs at the cut
        np.testing.assert_array_equal(got[l][0], exp[l][0], err_msg=f"vertices {l}")
        np.testing.assert_array_equal(got[l][1], exp[l][1], err_msg=f"edges {l}")
