"""The continuous-batching request loop (brook_b200.serving).

CPU tests drive the loop with a stand-in for skeletonize_batch that records what ran together and
how much device memory was held; the GPU test checks that every request's skeletons are the same
whether it runs alone or in a mix with others."""
import threading
import time

import numpy as np
import pytest

from brook_b200 import serving


class FakeBatch:
    """Records batches and the device bytes in flight; each batch takes `seconds`."""

    def __init__(self, seconds=0.05, fail_on=None):
        self.seconds = seconds
        self.fail_on = fail_on
        self.lock = threading.Lock()
        self.in_flight = 0
        self.peak = 0
        self.batches = []

    def __call__(self, volumes, output, **options):
        nbytes = sum(serving.footprint(v.shape, v.dtype) for v in volumes)
        with self.lock:
            self.in_flight += nbytes
            self.peak = max(self.peak, self.in_flight)
            self.batches.append([int(v.flat[0]) for v in volumes])
        time.sleep(self.seconds)
        with self.lock:
            self.in_flight -= nbytes
        if self.fail_on is not None and any(int(v.flat[0]) == self.fail_on for v in volumes):
            raise RuntimeError("planted failure")
        return [("result", int(v.flat[0])) for v in volumes]


@pytest.fixture
def fake(monkeypatch):
    f = FakeBatch()
    monkeypatch.setattr(serving, "skeletonize_batch", f)
    return f


def volume(tag, edge=16, dtype=np.uint32):
    v = np.zeros((edge, edge, edge), dtype)
    v.flat[0] = tag
    return v


def test_footprint_counts_labels_and_state():
    assert serving.footprint((10, 10, 10), np.uint64) == 1000 * (8 + serving.STATE_BYTES_PER_VOXEL)
    assert serving.footprint((10, 10, 10), np.uint8) == 1000 * (1 + serving.STATE_BYTES_PER_VOXEL)


def test_every_request_gets_its_own_result(fake):
    with serving.Server(workers=2) as server:
        futures = [server.submit(volume(i)) for i in range(1, 21)]
        results = [f.result(timeout=30) for f in futures]
    assert results == [("result", i) for i in range(1, 21)]
    assert sorted(t for b in fake.batches for t in b) == list(range(1, 21))


def test_requests_arriving_during_a_batch_join_a_later_one(fake):
    fake.seconds = 0.2
    with serving.Server(workers=2) as server:
        first = server.submit(volume(1))
        time.sleep(0.05)  # the first batch is running
        later = [server.submit(volume(i)) for i in range(2, 6)]
        for f in [first] + later:
            f.result(timeout=30)
    assert fake.batches[0] == [1]
    # the later arrivals ran on the free worker while the first batch was still running
    assert sorted(t for b in fake.batches[1:] for t in b) == [2, 3, 4, 5]
    assert later[0].request.started < first.request.finished


def test_memory_cap_bounds_what_is_in_flight(fake):
    per = serving.footprint((16, 16, 16), np.uint32)
    with serving.Server(workers=3, memory_cap=3 * per) as server:
        futures = [server.submit(volume(i)) for i in range(1, 13)]
        for f in futures:
            f.result(timeout=30)
    assert fake.peak <= 3 * per
    assert all(len(b) <= 3 for b in fake.batches)


def test_oversized_request_is_refused(fake):
    with serving.Server(memory_cap=1000) as server:
        with pytest.raises(ValueError, match="memory cap"):
            server.submit(volume(1))


def test_a_failed_batch_fails_its_requests_only(fake):
    fake.fail_on = 3
    fake.seconds = 0.01
    with serving.Server(workers=1, max_batch=1) as server:
        futures = [server.submit(volume(i)) for i in range(1, 6)]
        outcomes = [f.exception(timeout=30) for f in futures]
    assert [o is None for o in outcomes] == [True, True, False, True, True]


def test_replay_counts_latency_from_the_scheduled_arrival(fake):
    fake.seconds = 0.02
    requests = [(0.01 * i, volume(i + 1)) for i in range(8)]
    done = serving.replay(requests, lambda: serving.Server(workers=2))
    assert len(done) == 8
    assert all(r.latency >= 0.02 for r in done)
    p = serving.percentiles([r.latency for r in done])
    assert p["p50"] <= p["p99"]


@pytest.mark.gpu
def test_results_are_the_same_alone_and_in_a_mix(gpu):
    import brook_b200
    from brook_b200 import synthetic

    params = dict(scale=1.5, const=300, pdrf_scale=100000, pdrf_exponent=4)
    opts = dict(teasar_params=params, anisotropy=(16, 16, 40), dust_threshold=100)
    rng = np.random.default_rng(4)
    vols = []
    for i in range(12):
        shape = tuple(int(x) for x in rng.integers(32, 96, size=3))
        dtype = np.uint32 if i % 2 else np.uint64
        vols.append(synthetic.tube_volume(shape, objects=int(rng.integers(1, 5)), rng=rng, dtype=dtype))
    alone = [brook_b200.skeletonize(v, output="packed", **opts) for v in vols]
    with serving.Server(workers=2, **opts) as server:
        futures = [server.submit(v) for v in vols]
        mixed = [f.result(timeout=300) for f in futures]
    assert max(server.batches) > 1  # some requests really ran together
    for a, m in zip(alone, mixed):
        np.testing.assert_array_equal(a.labels, m.labels)
        np.testing.assert_array_equal(a.v_off, m.v_off)
        np.testing.assert_array_equal(a.vertices, m.vertices)
        np.testing.assert_array_equal(a.edges, m.edges)
        np.testing.assert_array_equal(a.radii, m.radii)
