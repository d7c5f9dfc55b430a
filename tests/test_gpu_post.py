"""Canonical post-processing on the device (brook_postprocess_canonical / brook_postprocess_step /
brook_skeleton_components through brook_b200.device_post) against the oracle (oracle/post.cpp),
bit for bit: every step alone and the whole chain, on seeded random sets with every kind of
cycle, tick and near component, on skeletonize's own output and on merged chunk fragments."""
import numpy as np
import pytest

from oracle import post as opost
from post_cases import assert_same_packed, from_packed, packed_set, to_packed

pytestmark = pytest.mark.gpu

STEPS = [("remove_dust", 60.0), ("remove_dust", 400.0), ("remove_loops", 0.0), ("join_components", 0.0),
         ("remove_ticks", 30.0), ("remove_ticks", 200.0), ("prune_unused", 0.0)]


def device_step(p, step, threshold):
    from brook_b200 import device_post as dp

    fn = {"remove_dust": lambda q: dp.remove_dust(q, threshold), "remove_loops": dp.remove_loops,
          "join_components": dp.join_close_components, "remove_ticks": lambda q: dp.remove_ticks(q, threshold),
          "prune_unused": dp.prune_unused}[step]
    return from_packed(fn(to_packed(p)))


def test_reference_known_answers_on_device(gpu):
    from brook_b200 import device_post as dp

    v = np.array([[0, 0, 0], [1, 0, 0], [5, 0, 0], [11, 0, 0]], np.float32)
    skel = dict(labels=np.array([1337]), vertex_offsets=np.array([0, 4]), edge_offsets=np.array([0, 2]), vertices=v,
                edges=np.array([[0, 1], [2, 3]], np.uint32), radii=np.full(4, 100, np.float32))
    joined = from_packed(dp.join_close_components(to_packed(skel)))
    np.testing.assert_array_equal(joined["edges"], [[0, 1], [1, 2], [2, 3]])
    done = from_packed(dp.postprocess(to_packed(skel), 0, 0))
    np.testing.assert_array_equal(done["edges"], [[0, 1], [1, 2], [2, 3]])
    gone = from_packed(dp.postprocess(to_packed(skel), 1000, 0))
    assert list(gone["labels"]) == [1337] and list(gone["vertex_offsets"]) == [0, 0]


@pytest.mark.parametrize("oriented", [True, False])
@pytest.mark.parametrize("seed", range(8))
def test_each_step_matches_oracle(gpu, seed, oriented):
    p = packed_set(seed, oriented=oriented)
    for step, t in STEPS:
        assert_same_packed(device_step(p, step, t), opost.run(p, step, t), f"{step}({t}) seed {seed}")


@pytest.mark.parametrize("seed", range(8))
def test_postprocess_matches_oracle(gpu, seed):
    from brook_b200 import device_post as dp

    p = packed_set(100 + seed, labels=12, max_components=6, max_size=120, cycles=6)
    for dust, ticks in ((0, 0), (60, 40), (400, 300)):
        got = from_packed(dp.postprocess(to_packed(p), dust, ticks))
        assert_same_packed(got, opost.postprocess(p, dust, ticks), f"postprocess({dust}, {ticks}) seed {seed}")


def test_large_components_match_oracle(gpu):
    """Components of thousands of vertices with dozens of cycles (the peeled walker's case)."""
    from brook_b200 import device_post as dp

    p = packed_set(7, labels=4, max_components=3, max_size=4000, cycles=40)
    for step, t in STEPS:
        assert_same_packed(device_step(p, step, t), opost.run(p, step, t), f"{step}({t})")
    assert_same_packed(from_packed(dp.postprocess(to_packed(p), 200, 300)), opost.postprocess(p, 200, 300), "chain")


def test_components_and_device_input(gpu):
    import torch

    from brook_b200 import device_post as dp

    p = packed_set(3)
    comps = dp.components(to_packed(p))
    assert comps.is_cuda and comps.dtype == torch.int64
    np.testing.assert_array_equal(comps.cpu().numpy(), opost.run(p, "components"))
    on_device = to_packed(p).to_device()
    assert on_device.on_device
    assert_same_packed(from_packed(dp.postprocess(on_device, 60, 40)), opost.postprocess(p, 60, 40), "device input")


def test_skeletonize_output_postprocess(gpu):
    import brook_b200 as bk
    from brook_b200 import device_post as dp
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((96, 96, 64), objects=12, seed=5)
    params = dict(scale=1.5, const=300, pdrf_scale=100000, pdrf_exponent=4)
    packed = bk.skeletonize(labels, teasar_params=params, anisotropy=(8, 8, 40), dust_threshold=0,
                            output="packed_device")
    host = from_packed(packed)
    got = from_packed(dp.postprocess(packed, 1500, 3500))
    assert_same_packed(got, opost.postprocess(host, 1500, 3500), "skeletonize output")


def test_chunked_postprocess(gpu):
    import brook_b200 as bk
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((80, 72, 48), objects=6, seed=9)
    params = dict(scale=1.5, const=300, pdrf_scale=100000, pdrf_exponent=4)
    opts = dict(chunk_shape=(40, 40, 48), overlap=1, teasar_params=params, anisotropy=(8, 8, 40), dust_threshold=0)
    merged = from_packed(bk.skeletonize_chunked(labels, output="packed", **opts))
    post = dict(dust_threshold=500, tick_threshold=800)
    got = from_packed(bk.skeletonize_chunked(labels, output="packed", postprocess=post, **opts))
    assert_same_packed(got, opost.postprocess(merged, 500, 800), "chunked")


def test_degenerate_inputs(gpu):
    """Empty sets, empty labels, isolated vertices, self loops and duplicate edges in both
    orientations: every step answers as the oracle does (no zero-size launch, no error)."""
    from brook_b200 import device_post as dp

    def packed(vs, es, labels):
        voff, eoff, verts, edges, radii = [0], [0], [], [], []
        for v, e in zip(vs, es):
            verts += v
            edges += e
            radii += [2.0] * len(v)
            voff.append(voff[-1] + len(v))
            eoff.append(eoff[-1] + len(e))
        return dict(labels=np.asarray(labels, np.int64), vertex_offsets=np.asarray(voff, np.int64),
                    edge_offsets=np.asarray(eoff, np.int64), vertices=np.asarray(verts, np.float32).reshape(-1, 3),
                    edges=np.asarray(edges, np.uint32).reshape(-1, 2), radii=np.asarray(radii, np.float32))

    tri = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [5, 5, 0]]
    cases = [
        packed([], [], []),                                                   # no labels
        packed([[]], [[]], [4]),                                              # one empty label
        packed([[[0, 0, 0]]], [[]], [4]),                                     # one isolated vertex
        packed([tri, []], [[[0, 1], [1, 2], [2, 0], [0, 0]], []], [4, 9]),    # a self loop beside a cycle
        packed([tri], [[[0, 1], [1, 0], [1, 2], [2, 1], [2, 0]]], [7]),       # duplicates, both orientations
        packed([tri, tri], [[[0, 1]], [[2, 3]]], [1, 2]),                     # vertices on no edge
    ]
    for i, p in enumerate(cases):
        for step, t in STEPS:
            assert_same_packed(device_step(p, step, t), opost.run(p, step, t), f"case {i} {step}({t})")
        assert_same_packed(from_packed(dp.postprocess(to_packed(p), 1, 1)), opost.postprocess(p, 1, 1), f"case {i}")
