"""The post-processing oracle (oracle/post.cpp) against the reference's own known answers and
hand-worked cases of each rule, plus invariants on seeded random sets (CPU only)."""
import numpy as np
import pytest

from oracle import post
from post_cases import packed_set


def one(vertices, edges, radii, label=1337):
    vertices = np.asarray(vertices, np.float32).reshape(-1, 3)
    edges = np.asarray(edges, np.uint32).reshape(-1, 2)
    return dict(labels=np.array([label], np.int64), vertex_offsets=np.array([0, len(vertices)], np.int64),
                edge_offsets=np.array([0, len(edges)], np.int64), vertices=vertices, edges=edges,
                radii=np.asarray(radii, np.float32))


def test_reference_known_answers():
    # tests/python/test_package.py:79-89 and cpp/tests/cpu_post_smoke.cpp:10-30 of the reference:
    # four collinear vertices in two pieces, radii 100
    skel = one([[0, 0, 0], [1, 0, 0], [5, 0, 0], [11, 0, 0]], [[0, 1], [2, 3]], np.full(4, 100))
    joined = post.run(skel, "join_components")
    np.testing.assert_array_equal(joined["edges"], [[0, 1], [1, 2], [2, 3]])
    processed = post.postprocess(skel, 0, 0)
    np.testing.assert_array_equal(processed["edges"], [[0, 1], [1, 2], [2, 3]])
    assert list(processed["labels"]) == [1337]
    gone = post.postprocess(skel, 1000, 0)  # 7 units of cable: dust
    assert list(gone["labels"]) == [1337] and list(gone["vertex_offsets"]) == [0, 0]


def test_loop_rules():
    # a lone triangle (no branch node) goes, and its vertices with it
    tri = one([[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 1], [1, 2], [2, 0]], np.ones(3))
    out = post.run(tri, "remove_loops")
    assert list(out["vertex_offsets"]) == [0, 0] and len(out["edges"]) == 0
    # one branch node: the cycle is replaced by an edge to its farthest node (ties to the lower)
    tail = one([[0, 0, 0], [1, 0, 0], [0, 1, 0], [-1, -1, 0], [-2, -2, 0]],
               [[0, 1], [1, 2], [2, 0], [0, 3], [3, 4]], np.ones(5))
    np.testing.assert_array_equal(post.run(tail, "remove_loops")["edges"], [[0, 1], [0, 3], [3, 4]])
    # two branch nodes on a square with two tails: the search from 0 closes the cycle 0-3-2-1-0,
    # the branch nodes sit at path positions 1 and 3 of 4, so the side through node 1 goes
    sq = one([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [-1, 0, 0], [2, 1, 0]],
             [[0, 1], [1, 2], [2, 3], [3, 0], [0, 4], [2, 5]], np.ones(6))
    np.testing.assert_array_equal(post.run(sq, "remove_loops")["edges"], [[0, 3], [0, 4], [2, 3], [2, 5]])
    # a self loop: the triangle through node 0 (a branch node by its four row ends) becomes the
    # edge to its farthest node, then the search meets the self loop (a one-node cycle), which
    # ends the rounds; self loops never reach the output
    self_loop = one([[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 0], [0, 1], [1, 2], [2, 0]], np.ones(3))
    np.testing.assert_array_equal(post.run(self_loop, "remove_loops")["edges"], [[0, 1]])


def test_tick_rule():
    # a long trunk with one short branch: the short branch goes, the trunk stays
    v = [[0, 0, 0], [10, 0, 0], [20, 0, 0], [30, 0, 0], [10, 1, 0]]
    t = one(v, [[0, 1], [1, 2], [2, 3], [1, 4]], np.ones(5))
    out = post.run(t, "remove_ticks", 5.0)
    np.testing.assert_array_equal(out["edges"], [[0, 1], [1, 2], [2, 3]])
    assert list(post.run(t, "remove_ticks", 0.5)["edge_offsets"]) == [0, 4]  # nothing is that short


def _components(p, label):
    v0, v1 = p["vertex_offsets"][label], p["vertex_offsets"][label + 1]
    e = p["edges"][p["edge_offsets"][label]:p["edge_offsets"][label + 1]].astype(np.int64)
    parent = list(range(v1 - v0))

    def find(x):
        while parent[x] != x:
            x = parent[x]
        return x

    for a, b in e:
        ra, rb = find(a), find(b)
        if ra != rb:
            parent[max(ra, rb)] = min(ra, rb)
    return {find(i) for i in range(v1 - v0) if any(i in (a, b) for a, b in e)}, len(e)


@pytest.mark.parametrize("seed", range(6))
def test_invariants_on_random_sets(seed):
    p = packed_set(seed)
    loops = post.run(p, "remove_loops")
    for l in range(len(loops["labels"])):
        comps, ne = _components(loops, l)
        used = {int(x) for x in loops["edges"][loops["edge_offsets"][l]:loops["edge_offsets"][l + 1]].ravel()}
        assert ne == len(used) - len(comps)  # a forest: edges = vertices on edges - trees
    joined = post.run(loops, "join_components")
    for l in range(len(joined["labels"])):
        assert len(_components(joined, l)[0]) <= max(len(_components(loops, l)[0]), 1)
    done = post.postprocess(p, 30, 60)
    assert list(done["labels"]) == list(p["labels"])
    comps = post.run(p, "components")
    assert len(comps) == len(p["radii"]) and np.all(comps <= np.arange(len(comps)))
