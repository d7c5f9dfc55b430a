"""Chunks and the merge of fragments against the oracle: brook_merge_skeletons (the reference's
merge_parts, packed_merge.cu:88-166) on the device and its restatement oracle/merge.py give the
same packed skeletons, bit for bit; skeletonize_chunked equals the oracle run chunk by chunk and
merged."""
import numpy as np
import pytest

from oracle import merge as om
from oracle import oracle
from test_gpu_parity import CFG0_PARAMS, bk

pytestmark = pytest.mark.gpu

OPTS = dict(teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100)


def _same(packed, exp, what):
    np.testing.assert_array_equal(packed.labels, exp["labels"], err_msg=f"labels {what}")
    np.testing.assert_array_equal(packed.v_off, exp["vertex_offsets"], err_msg=f"vertex offsets {what}")
    np.testing.assert_array_equal(packed.e_off, exp["edge_offsets"], err_msg=f"edge offsets {what}")
    np.testing.assert_array_equal(packed.vertices, exp["vertices"], err_msg=f"vertices {what}")
    np.testing.assert_array_equal(packed.edges, exp["edges"], err_msg=f"edges {what}")
    np.testing.assert_array_equal(packed.radii.view(np.uint32), exp["radii"].view(np.uint32), err_msg=f"radii {what}")


def _chunks(labels, chunk, overlap):
    from brook_b200 import chunked, sharding

    slices = list(sharding.iter_chunks(labels.shape, chunk, overlap))
    origins = chunked.physical_origins([[s.start for s in sl] for sl in slices], OPTS["anisotropy"])
    return [np.asfortranarray(labels[sl]) for sl in slices], origins


def test_merge_fragments_matches_oracle(gpu):
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((96, 80, 48), objects=10, seed=8)
    chunks, origins = _chunks(labels, (56, 48, 48), 8)
    assert len(chunks) == 4
    parts = [bk().skeletonize(c, output="packed", fix_borders=True, **OPTS) for c in chunks]
    exp = om.merge([oracle.skeletonize(c, threads=8, fix_borders=True, **OPTS).packed() for c in chunks], origins)
    assert len(exp["labels"]) >= 8
    _same(bk().merge_fragments(parts, origins), exp, "host parts")
    dev = [bk().skeletonize(c, output="packed_device", fix_borders=True, **OPTS) for c in chunks]
    merged = bk().merge_fragments(dev, origins, on_device=True)
    assert merged.on_device
    _same(merged.to_host(), exp, "device parts")


@pytest.mark.parametrize("budget", [None, 1])
def test_skeletonize_chunked_matches_oracle(gpu, budget):
    """All chunks in one batch, or one chunk per call (a budget of 1 byte)."""
    from brook_b200 import synthetic

    labels = synthetic.dense_volume((128, 96, 64), seeds=30, seed=6, dtype=np.uint32)
    chunks, origins = _chunks(labels, (64, 64, 64), 1)
    exp = om.merge([oracle.skeletonize(c, threads=8, fix_borders=True, **OPTS).packed() for c in chunks], origins)
    got = bk().skeletonize_chunked(labels, chunk_shape=(64, 64, 64), overlap=1, output="packed", memory_budget=budget,
                                   **OPTS)
    assert len(got) > 10
    _same(got, exp, f"chunked budget={budget}")
