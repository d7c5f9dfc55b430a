"""The Python argument surface's host-side rules (no GPU): TEASAR defaults, label formatting and the
options refused before any device call. They follow the reference's src/brook/_intake.py:23-37
(format_labels) and its kimimaro.trace defaults for omitted keys (skeleton.hpp:23-27)."""
import numpy as np
import pytest

import brook_b200
from brook_b200 import _intake


def test_omitted_teasar_keys_take_the_trace_defaults():
    p = _intake.teasar({"scale": 2, "const": 5})
    assert p["scale"] == 2.0 and p["const"] == 5.0
    assert p["pdrf_exponent"] == 16.0 and p["pdrf_scale"] == 5000.0  # kimimaro.trace, not DEFAULT_TEASAR_PARAMS
    assert p["soma_detection_threshold"] == 1100.0 and p["max_paths"] is None
    assert isinstance(p["const"], float)
    assert _intake.teasar({"max_paths": 3})["max_paths"] == 3


def test_unknown_teasar_key_is_refused():
    with pytest.raises(TypeError, match="unexpected TEASAR parameter"):
        _intake.teasar({"scale": 1, "tolerance": 2})


def test_default_params_are_the_references():
    assert brook_b200.DEFAULT_TEASAR_PARAMS == {
        "scale": 1.5, "const": 300, "pdrf_scale": 100000, "pdrf_exponent": 4, "soma_acceptance_threshold": 3500,
        "soma_detection_threshold": 750, "soma_invalidation_const": 300, "soma_invalidation_scale": 2}


def test_format_labels_keeps_the_bytes():
    a = np.asfortranarray(np.arange(24, dtype=np.uint16).reshape(2, 3, 4))
    f = _intake.format_labels(a)
    assert f.shape == (2, 3, 4) and np.shares_memory(f, a) and f.flags.f_contiguous
    b = np.zeros((5, 6), bool)
    b[1, 2] = True
    g = _intake.format_labels(b)
    assert g.dtype == np.uint8 and g.shape == (5, 6, 1) and np.shares_memory(g, b) and g[1, 2, 0] == 1
    assert _intake.format_labels(np.ones(7, np.int32)).shape == (7, 1, 1)
    assert _intake.format_labels(np.ones((3, 4, 5, 1, 1), np.uint64)).shape == (3, 4, 5)


def test_format_labels_refuses_what_the_path_cannot_take():
    with pytest.raises(_intake.DimensionError):
        _intake.format_labels(np.ones((2, 3, 4, 2), np.uint32))
    with pytest.raises(TypeError):
        _intake.format_labels(np.ones((2, 3, 4), np.float32))


def test_options_outside_the_path_raise_before_any_device_call():
    v = np.ones((4, 4, 4), np.uint32)
    with pytest.raises(ValueError, match="output"):
        brook_b200.skeletonize(v, output="dense")
    for option in ({"voxel_graph": np.zeros((4, 4, 4), np.uint32)},):
        with pytest.raises(NotImplementedError):
            brook_b200.skeletonize(v, **option)
    with pytest.raises(ValueError, match="output"):
        brook_b200.skeletonize_batch([v], output="dense")


def test_a_volume_within_the_dust_threshold_is_empty_without_a_device():
    v = np.ones((4, 4, 4), np.uint32)  # 64 voxels <= dust 1000: nothing to trace
    assert brook_b200.skeletonize(v) == {}
    p = brook_b200.skeletonize(v, output="packed", anisotropy=(2, 2, 2))
    assert len(p) == 0 and p.anisotropy == (2.0, 2.0, 2.0)


def test_streaming_selection_rule(monkeypatch):
    """streaming as given, else BROOK_STREAMING, else the in-core footprint rule (small volumes stay
    in-core without asking the device)."""
    from brook_b200 import _intake

    small = np.zeros((8, 8, 8), np.uint32)
    monkeypatch.delenv("BROOK_STREAMING", raising=False)
    assert _intake._use_streaming(True, small, 0) and not _intake._use_streaming(False, small, 0)
    assert not _intake._use_streaming(None, small, 0)
    for value, expected in (("1", True), ("on", True), ("0", False), ("off", False), ("no", False)):
        monkeypatch.setenv("BROOK_STREAMING", value)
        assert _intake._use_streaming(None, small, 0) is expected
    assert _intake._use_streaming(False, small, 0) is False
