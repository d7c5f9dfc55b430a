"""The option surface beyond the defaults, against the oracle: fix_branching=False (one SSSP from
the root kept per object, every path walked back to the root; trace.cu:151-160,
batched_regular.inc:113-152) and a PDRF exponent that is not a power of two (the reference's powf,
trace_primitives.cu:119-129; only odd integers are refused, skeletonize.cu:101-103)."""
import os
import tempfile

import numpy as np
import pytest

from oracle import oracle
from test_gpu_parity import CFG0_PARAMS, assert_same, bk

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [0, 1])
def test_fix_branching_off_matches_oracle(gpu, seed):
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((72, 64, 56), objects=8, seed=seed)
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100, fix_branching=False)
    got = bk().skeletonize(labels, output="packed", **opts)
    exp = oracle.skeletonize(labels, threads=8, **opts)
    assert len(got) > 0
    assert_same(got, exp, f"fix_branching=False seed {seed}")
    on = oracle.skeletonize(labels, threads=8, **dict(opts, fix_branching=True))
    assert not np.array_equal(on.array("vertices"), exp.array("vertices"))  # the option changes the skeletons


def test_fix_branching_off_dense_cells_clusters_and_batch(gpu, monkeypatch):
    """Dense cells (large objects on thread-block clusters) and an uneven batch, branching off."""
    from brook_b200 import synthetic

    labels = synthetic.dense_volume((128, 128, 96), seeds=30, seed=5)
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(8, 8, 40), dust_threshold=100, fix_branching=False)
    assert_same(bk().skeletonize(labels, output="packed", **opts), oracle.skeletonize(labels, threads=8, **opts),
                "dense cells")
    monkeypatch.setenv("BROOK_B200_PREPARE_CLUSTER_VOXELS", "1")
    monkeypatch.setenv("BROOK_B200_TRACE_CLUSTER_VOXELS", "1")
    samples = [synthetic.tube_volume(shape, objects=6, seed=s)
               for s, shape in enumerate([(64, 48, 40), (40, 56, 64), (48, 48, 48)])]
    batch = bk().skeletonize_batch(samples, output="packed", **opts)
    for i, v in enumerate(samples):
        assert_same(batch[i], oracle.skeletonize(v, threads=8, **opts), f"batch sample {i} on clusters")


def _gpu_fields(labels, monkeypatch, **opts):
    """The skeletons and the prepared PDRF field of one call (BROOK_B200_DUMP_FIELDS)."""
    folder = tempfile.mkdtemp()
    prefix = os.path.join(folder, "fields")
    monkeypatch.setenv("BROOK_B200_DUMP_FIELDS", prefix)
    got = bk().skeletonize(labels, output="packed", **opts)
    monkeypatch.delenv("BROOK_B200_DUMP_FIELDS")
    pdrf = np.fromfile(prefix + ".pdrf", np.float32).reshape(labels.shape, order="F")
    return got, pdrf


@pytest.mark.parametrize("exponent,fix_branching", [(6, True), (2.5, True), (12, False)])
def test_pdrf_exponent_not_a_power_of_two(gpu, monkeypatch, exponent, fix_branching):
    """The PDRF with powf is within 1e-6 relative of the oracle's float64 power (CUDA's powf is
    not correctly rounded, so the bits may differ); traced from the GPU's own field, the oracle
    gives the GPU's skeletons bit for bit."""
    from brook_b200 import synthetic

    labels = synthetic.tube_volume((64, 64, 48), objects=6, seed=2)
    params = dict(CFG0_PARAMS, pdrf_exponent=exponent)
    opts = dict(teasar_params=params, anisotropy=(16, 16, 40), dust_threshold=100, fix_branching=fix_branching)
    got, pdrf = _gpu_fields(labels, monkeypatch, **opts)
    exp = oracle.skeletonize(labels, threads=8, stages=True, **opts)
    ref = exp.field("pdrf")
    finite = np.isfinite(ref) & (pdrf != 0) & (ref != 0)  # object voxels but the root rails
    assert finite.sum() > 1000
    np.testing.assert_allclose(pdrf[finite], ref[finite], rtol=1e-6, atol=0)
    traced = oracle.skeletonize(labels, threads=8, pdrf_field=pdrf, **opts)
    assert len(got) > 0
    assert_same(got, traced, f"exponent {exponent}")
    with pytest.raises(Exception, match="odd"):
        bk().skeletonize(labels, output="packed", **dict(opts, teasar_params=dict(params, pdrf_exponent=3)))


def test_engine_graph_matches_eager_launches(gpu, monkeypatch):
    """The engine's launches (prepare, target orders, trace) run as one CUDA graph per call; the
    context updates its executable graph in place for the next call. The skeletons equal those of
    the same launches made one by one (BROOK_B200_GRAPH=0) and the oracle's."""
    from brook_b200 import _native, synthetic

    labels = synthetic.tube_volume((64, 64, 64), objects=8, seed=9)
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100)
    first = bk().skeletonize(labels, output="packed", **opts)
    stats = _native.stats()
    assert stats["graph_launches"] == 1 and stats["ms_trace"] > 0 and stats["ms_prepare"] > 0
    second = bk().skeletonize(labels, output="packed", **opts)
    assert _native.stats().get("graph_updates", 0) + _native.stats().get("graph_instantiations", 0) == 1
    monkeypatch.setenv("BROOK_B200_GRAPH", "0")
    eager = bk().skeletonize(labels, output="packed", **opts)
    assert "graph_launches" not in _native.stats()
    exp = oracle.skeletonize(labels, threads=8, **opts)
    for got in (first, second, eager):
        assert_same(got, exp, "graph / eager")


def test_autotune_installs_a_choice_that_keeps_the_skeletons(gpu, monkeypatch, tmp_path):
    """brook_b200.tuning.autotune measures launch choices on the caller's volumes, installs the
    fastest for their workload class and saves it; a new context loads it; the skeletons do not
    depend on the choice."""
    from brook_b200 import _native, synthetic, tuning

    monkeypatch.setenv("BROOK_B200_TUNING_CACHE", str(tmp_path / "tuning.json"))
    labels = synthetic.tube_volume((96, 96, 64), objects=12, seed=5)
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100)
    result = tuning.autotune(labels, **opts)
    assert result["engine_ms"] > 0 and result["tuning"]["trace_cluster_ctas"] in (0, 4, 8)
    saved = tuning._read()
    assert any(result["workload_class"] in entries for entries in saved.values())
    got = bk().skeletonize(labels, output="packed", **opts)
    assert_same(got, oracle.skeletonize(labels, threads=8, **opts), "tuned")
    # every candidate choice gives the same skeletons
    for ctas, percent in ((8, 0), (4, 25)):
        t = _native.Tuning(ctas, 1, 1, percent)
        ctx = _native.context(0)
        _native.check(_native.load().brook_context_set_tuning(ctx, int(result["workload_class"], 16), t))
        assert_same(bk().skeletonize(labels, output="packed", **opts),
                    oracle.skeletonize(labels, threads=8, **opts), f"choice {ctas}/{percent}")
    _native.check(_native.load().brook_context_set_tuning(_native.context(0), int(result["workload_class"], 16), None))
