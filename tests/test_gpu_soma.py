"""Somata against the oracle (trace.cu:98-131, soma.cu:141-237): an object whose DBF maximum
passes soma_detection_threshold is prepared and traced in a crop of its own, its voids filled and
its DBF recomputed when anything was filled; past soma_acceptance_threshold it is a soma: the root
at the maximum nearest the maxima's centroid, the DAF seeded through free space, the soma's ball
invalidated first, every path trimmed to the soma radius."""
import numpy as np
import pytest

from oracle import oracle
from test_gpu_parity import assert_same, bk
from test_oracle_golden import SOMA_PARAMS, _components, _soma_with_processes

pytestmark = pytest.mark.gpu


def _both(labels, **opts):
    got = bk().skeletonize(labels, output="packed", **opts)
    exp = oracle.skeletonize(labels, threads=8, **opts)
    return got, exp


@pytest.mark.parametrize("fix_branching", [True, False])
@pytest.mark.parametrize("hollow", [False, True])
def test_soma_matches_oracle(gpu, fix_branching, hollow):
    labels = _soma_with_processes()
    if hollow:
        labels[33:40, 30:34, 33:40] = 0
    opts = dict(teasar_params=SOMA_PARAMS, dust_threshold=0, fix_branching=fix_branching, fix_borders=False)
    got, exp = _both(labels, **opts)
    assert_same(got, exp, f"soma fix_branching={fix_branching} hollow={hollow}")
    sk = got.to_skeletons()[1]
    assert np.any(np.all(sk.vertices == 36, axis=1)) and _components(sk.vertices, sk.edges) == 1
    assert bk()._native.stats()["somata"] == 1


def test_somata_among_other_objects(gpu):
    """Two somata (one with a void that encloses another label, which is traced on its own), a
    candidate below the acceptance threshold, thin objects, border targets on, anisotropy."""
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((96, 88, 72), objects=8, seed=4, radius=(1.5, 3.0)).astype(np.uint32)
    grid = np.indices(labels.shape)
    for label, centre, radius in ((21, (30, 30, 30), 11), (22, (70, 60, 40), 9), (23, (60, 20, 55), 6)):
        ball = sum((g - c) ** 2 for g, c in zip(grid, centre)) <= radius ** 2
        labels[ball] = label
    labels[26:34, 27:33, 28:32] = 0       # a void in soma 21 ...
    labels[29:31, 29:31, 29:31] = 30      # ... holding a small object of another label
    labels[30, 0:30, 30] = 21             # a process of soma 21 out to the volume's face
    # global DBF maxima: 21 6.25 (its void lowers it), 22 9.06, 23 6.08; the tubes at most 4.3
    params = dict(SOMA_PARAMS, soma_detection_threshold=5.5, soma_acceptance_threshold=8.5)
    for fix_branching in (True, False):
        opts = dict(teasar_params=params, anisotropy=(1, 1, 1.25), dust_threshold=5, fix_branching=fix_branching)
        got, exp = _both(np.asfortranarray(labels), **opts)
        assert {21, 22, 23} <= set(got.labels.tolist())
        assert_same(got, exp, f"somata fix_branching={fix_branching}")
    stats = bk()._native.stats()
    assert stats["soma_candidates"] == 3 and stats["somata"] == 2


def test_somata_in_a_batch_and_on_clusters(gpu, monkeypatch):
    """Soma samples inside an uneven batch (each result equals the oracle on its sample), with
    every object on a thread-block cluster."""
    from brook_b200 import synthetic

    monkeypatch.setenv("BROOK_B200_PREPARE_CLUSTER_VOXELS", "1")
    monkeypatch.setenv("BROOK_B200_TRACE_CLUSTER_VOXELS", "1")
    samples = [_soma_with_processes(), synthetic.tube_volume((48, 40, 56), objects=5, seed=1),
               _soma_with_processes(size=60, centre=30, radius=10)[:, :, 4:]]
    opts = dict(teasar_params=SOMA_PARAMS, dust_threshold=0, fix_borders=True)
    batch = bk().skeletonize_batch(samples, output="packed", **opts)
    for i, v in enumerate(samples):
        assert_same(batch[i], oracle.skeletonize(v, threads=8, **opts), f"sample {i}")
