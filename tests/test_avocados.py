"""fix_avocados: the avocado stage (avocado.cpp:223-239, which restates Kimimaro 5.8.1's
engage_avocado_protection). An object whose distance field passes soma_detection_threshold / 2.5
is a candidate; the rays from its crop's deepest voxel decide whether it is a pit inside another
object (the fruit), which then absorbs it; the stage runs up to 20 passes, refreshes the distance
field after a pass that merged, and renumbers the ids by first voxel. Candidates are taken in the
iteration order of a CPython set of ints.

Pinned here: the set order against this interpreter's own sets (CPython 3.12), and the stage and
skeletons against the answers the reference's tests hold from Kimimaro 5.8.1
(tests/python/test_package.py: the rule samples, the stage's mapping / first voxels / labels, the
anisotropic refresh, the unreachable cavity). The GPU tests check the CUDA path against the oracle."""
import sys

import numpy as np
import pytest

from oracle import oracle

RULE_PARAMS = dict(scale=1.5, const=1, pdrf_scale=100000, pdrf_exponent=4, soma_detection_threshold=4.5,
                   soma_acceptance_threshold=1e6, soma_invalidation_scale=1., soma_invalidation_const=0)
CAVITY_PARAMS = dict(scale=1.5, const=2, pdrf_scale=100000, pdrf_exponent=4, soma_detection_threshold=6,
                     soma_acceptance_threshold=8, soma_invalidation_scale=1., soma_invalidation_const=0)
REFRESH_ANISOTROPY = (1.1, 1.3, 2.0)


def rule_samples():
    """A pit (2) with two lobes, one inside a one-voxel shell (1) and one in the open, joined
    through a hole in the shell; the same with x and z swapped; three labels whose first voxels come
    in the order 3, 7, 5 (the reference's test_package.py:847-866)."""
    tie = np.zeros((16, 9, 16), np.uint32)
    tie[8:13, 1:6, 1:6] = 1
    tie[9:12, 2:5, 2:5] = 2
    tie[3:9, 2, 2] = 2
    tie[3, 2, 2:9] = 2
    tie[2:5, 2:5, 9:12] = 2
    order = np.zeros((16, 9, 16), np.uint32)
    order[0:3, 0:3, 10:13] = 5
    order[10:13, 0:3, 0:3] = 3
    order[5:8, 0:3, 5:8] = 7
    return [tie, np.ascontiguousarray(tie.transpose(2, 1, 0)), order]


RULE_KEYS = [[2], [2, 1], [3, 7, 5]]


def refresh_sample():
    sample = np.zeros((7, 7, 7), np.uint32)
    sample[1:6, 1:6, 1:6] = 1
    sample[2:5, 2:5, 2:5] = 2
    return sample


def cavity_samples():
    """A slab with a background cavity, a pit fully inside a fruit, a pit open to one face beside a
    cavity, two fruits with pits whose ids interleave (test_package.py:619-639)."""
    hole = np.zeros((40, 40, 40), np.uint32)
    hole[4:36, 4:36, 4:20] = 1
    hole[14:26, 14:26, 8:16] = 0
    hole[6:34, 30:34, 24:36] = 2
    avocado = np.zeros((40, 40, 40), np.uint32)
    avocado[2:38, 2:38, 2:30] = 3
    avocado[10:30, 10:30, 8:24] = 4
    avocado[4:36, 33:37, 31:39] = 5
    mixed = np.zeros((40, 40, 40), np.uint32)
    mixed[3:37, 3:37, 3:37] = 6
    mixed[8:20, 8:20, 3:15] = 7
    mixed[24:32, 24:32, 24:32] = 0
    two = np.zeros((40, 40, 40), np.uint16)
    two[2:38, 2:18, 2:38] = 8
    two[10:30, 6:14, 10:30] = 9
    two[2:38, 22:38, 2:38] = 10
    two[10:30, 26:34, 10:30] = 11
    return [hole, avocado, mixed, two]


def unreachable_cavity():
    labels = np.zeros((26, 39, 26), np.uint32)
    labels[2:24, 3:38, 1:23] = 1
    labels[8:18, 17:26, 9:16] = 0
    return np.asfortranarray(labels)


# ---- the set order ---------------------------------------------------------------------------------


@pytest.mark.skipif(sys.version_info[:2] != (3, 12), reason="the restatement follows CPython 3.12's sets")
@pytest.mark.parametrize("seed", range(12))
def test_set_order_matches_cpython(seed):
    rng = np.random.default_rng(seed)
    hi = int(rng.choice([16, 100, 5000, 200000]))
    A, B, ops = set(), set(), []
    for _ in range(int(rng.integers(50, 3000))):
        r = rng.random()
        k = int(rng.integers(0, hi))
        if r < 0.45:
            A.add(k); ops.append((0, k))
        elif r < 0.65:
            A.discard(k); ops.append((1, k))
        elif r < 0.9:
            B.add(k); ops.append((2, k))
        elif r < 0.95:
            A -= B; B = set(); ops.append((3, 0))
        elif r < 0.995:
            A |= B; B = set(); ops.append((4, 0))
        else:
            A = set(); ops.append((5, 0))
    assert oracle.pyset_order(ops) == list(A)


# ---- the stage and its skeletons against Kimimaro's answers ---------------------------------------


@pytest.mark.parametrize("fix_branching", [True, False])
def test_rule_samples_keep_kimimaros_labels(fix_branching):
    for sample, keys in zip(rule_samples(), RULE_KEYS):
        out = oracle.skeletonize(sample, RULE_PARAMS, dust_threshold=0, fix_branching=fix_branching,
                                 fix_avocados=True, threads=4)
        assert out.array("labels").tolist() == keys


def test_stage_mapping_first_voxels_and_labels():
    expected = [([0, 2], [168], {1: 1, 2: 1}, True),
                ([0, 2, 1], [329, 1169], {2: 1, 1: 2}, False),
                ([0, 3, 7, 5], [10, 725, 1440], {3: 1, 7: 2, 5: 3}, False)]
    for sample, (mapping, roots, ids, refreshed) in zip(rule_samples(), expected):
        out = oracle.skeletonize(sample, RULE_PARAMS, dust_threshold=0, fix_avocados=True, stages=True)
        assert out.array("mapping").tolist() == mapping
        assert out.array("cc_roots").tolist() == roots
        cc = out.field("cc")
        np.testing.assert_array_equal(cc, np.select([sample == k for k in ids], list(ids.values()), 0))
        plain_edt = oracle.edt(np.asfortranarray(cc))
        if refreshed:
            np.testing.assert_array_equal(out.field("dbf"), plain_edt)
        else:  # the input's own field
            first = oracle.edt(np.asfortranarray(oracle.skeletonize(sample, RULE_PARAMS, dust_threshold=0,
                                                                    stages=True).field("cc")))
            np.testing.assert_array_equal(out.field("dbf"), first)


def test_anisotropic_refresh_and_its_skeleton():
    sample = refresh_sample()
    params = dict(RULE_PARAMS, soma_detection_threshold=5)
    out = oracle.skeletonize(sample, params, REFRESH_ANISOTROPY, dust_threshold=0, fix_avocados=True, stages=True)
    assert out.array("mapping").tolist() == [0, 1] and out.array("cc_roots").tolist() == [57]
    np.testing.assert_array_equal(out.field("cc"), (sample > 0).astype(np.uint32))
    assert out.field("dbf")[3, 3, 2:5].view(np.uint32).tolist() == [0x40533334] * 3
    vertices = np.arange(1, 6, dtype=np.float32)[:, None] * np.array(REFRESH_ANISOTROPY, np.float32)
    radii = [0x3f8ccccd, 0x400ccccd, 0x40533334, 0x400ccccd, 0x3f8ccccd]
    for fix_branching in (True, False):
        skel = oracle.skeletonize(sample, params, REFRESH_ANISOTROPY, dust_threshold=0, fix_branching=fix_branching,
                                  fix_avocados=True).skeletons()
        assert list(skel) == [1]
        v, e, r = skel[1]
        np.testing.assert_array_equal(v, vertices)
        np.testing.assert_array_equal(e, [[0, 1], [1, 2], [2, 3], [3, 4]])
        assert r.view(np.uint32).tolist() == radii


def test_unreachable_cavity_stops_the_object():
    """The stage paints the slab's enclosed cavity without a merge, so the field is not refreshed and
    the painted voxels keep distance zero, an infinite penalty: a DAF target inside the cavity has
    no path to a rail and ends the object's tracing."""
    out = oracle.skeletonize(unreachable_cavity(), CAVITY_PARAMS, dust_threshold=10, fix_avocados=True)
    assert int(out.array("avocado_passes")[0]) == 1
    skel = out.skeletons()
    assert list(skel) == [1]
    v, e, _ = skel[1]
    assert len(v) - len(e) == 1


@pytest.mark.parametrize("fix_branching", [True, False])
def test_cavity_samples_run(fix_branching):
    for sample in cavity_samples():
        out = oracle.skeletonize(sample, CAVITY_PARAMS, dust_threshold=10, fix_branching=fix_branching,
                                 fix_avocados=True, threads=4)
        assert len(out.array("labels")) >= 1


# ---- the CUDA path ---------------------------------------------------------------------------------


def _gpu(labels, params, anisotropy=(1, 1, 1), **opts):
    import brook_b200
    from brook_b200 import _native

    got = brook_b200.skeletonize(labels, params, anisotropy, output="packed", fix_avocados=True, **opts)
    return got, _native.stats()


@pytest.mark.gpu
@pytest.mark.parametrize("fix_branching", [True, False])
def test_gpu_rule_samples_keep_kimimaros_labels(gpu, fix_branching):
    from test_gpu_parity import assert_same

    for sample, keys in zip(rule_samples(), RULE_KEYS):
        got, stats = _gpu(sample, RULE_PARAMS, dust_threshold=0, fix_branching=fix_branching)
        assert got.labels.tolist() == keys
        exp = oracle.skeletonize(sample, RULE_PARAMS, dust_threshold=0, fix_branching=fix_branching,
                                 fix_avocados=True, threads=4)
        assert stats["avocado_passes"] == int(exp.array("avocado_passes")[0])
        assert_same(got, exp, f"rule sample {keys}")


@pytest.mark.gpu
def test_gpu_anisotropic_refresh_skeleton(gpu):
    sample = refresh_sample()
    params = dict(RULE_PARAMS, soma_detection_threshold=5)
    vertices = np.arange(1, 6, dtype=np.float32)[:, None] * np.array(REFRESH_ANISOTROPY, np.float32)
    radii = [0x3f8ccccd, 0x400ccccd, 0x40533334, 0x400ccccd, 0x3f8ccccd]
    for fix_branching in (True, False):
        got, _ = _gpu(sample, params, REFRESH_ANISOTROPY, dust_threshold=0, fix_branching=fix_branching)
        assert got.labels.tolist() == [1]
        np.testing.assert_array_equal(got.vertices, vertices)
        np.testing.assert_array_equal(got.edges, [[0, 1], [1, 2], [2, 3], [3, 4]])
        assert np.asarray(got.radii, np.float32).view(np.uint32).tolist() == radii


@pytest.mark.gpu
def test_gpu_unreachable_cavity_and_cavity_samples(gpu):
    from test_gpu_parity import assert_same

    got, stats = _gpu(unreachable_cavity(), CAVITY_PARAMS, dust_threshold=10)
    assert stats["avocado_passes"] == 1 and stats["zero_distances"] > 0
    exp = oracle.skeletonize(unreachable_cavity(), CAVITY_PARAMS, dust_threshold=10, fix_avocados=True)
    assert_same(got, exp, "unreachable cavity")
    assert len(got.vertices) - len(got.edges) == 1
    for fix_branching in (True, False):
        for detection in (6, 1000):  # with and without somata
            params = dict(CAVITY_PARAMS, soma_detection_threshold=detection,
                          soma_acceptance_threshold=detection + 2)
            for i, sample in enumerate(cavity_samples()):
                got, _ = _gpu(sample, params, dust_threshold=10, fix_branching=fix_branching)
                exp = oracle.skeletonize(sample, params, dust_threshold=10, fix_branching=fix_branching,
                                         fix_avocados=True, threads=4)
                assert_same(got, exp, f"cavity sample {i} detection {detection} branching {fix_branching}")


@pytest.mark.gpu
def test_gpu_avocados_in_a_batch(gpu):
    import brook_b200
    from test_gpu_parity import assert_same

    samples = rule_samples() + cavity_samples()
    batch = brook_b200.skeletonize_batch(samples, CAVITY_PARAMS, output="packed", dust_threshold=10,
                                         fix_avocados=True, fill_holes=True)
    for i, sample in enumerate(samples):
        exp = oracle.skeletonize(sample, CAVITY_PARAMS, dust_threshold=10, fix_avocados=True, fill_holes=True,
                                 threads=4)
        assert_same(batch[i], exp, f"batch sample {i}")
