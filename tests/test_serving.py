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
    """Records batches and the device bytes held; each batch takes `seconds`.

    Like a library context, each worker thread keeps the blocks of its last batch for reuse
    (`keeps`) until it hands them back (`trim_context`); `state` is the per-voxel state a batch
    reports as its peak."""

    def __init__(self, seconds=0.05, fail_on=None, keeps=False, state=None):
        self.seconds = seconds
        self.fail_on = fail_on
        self.keeps = keeps
        self.state = state
        self.lock = threading.Lock()
        self.in_flight = 0
        self.kept = {}  # thread -> bytes kept after its last batch
        self.peak = 0
        self.batches = []
        self.trims = 0
        self.last = {}  # thread -> (kept, peak) of its last batch

    def held(self):
        return self.in_flight + sum(self.kept.values())

    def __call__(self, volumes, output, **options):
        me = threading.get_ident()
        nbytes = sum(serving.footprint(v.shape, v.dtype) for v in volumes)
        with self.lock:
            self.in_flight += nbytes
            self.peak = max(self.peak, self.held())
            self.batches.append([int(v.flat[0]) for v in volumes])
        time.sleep(self.seconds)
        with self.lock:
            self.in_flight -= nbytes
            if self.keeps:
                self.kept[me] = max(self.kept.get(me, 0), nbytes)
            voxels = sum(v.size for v in volumes)
            state = self.state if self.state is not None else serving.STATE_BYTES_PER_VOXEL
            peak = sum(v.nbytes for v in volumes) + voxels * state + serving.REQUEST_BYTES * len(volumes)
            self.last[me] = (self.kept.get(me, 0), peak)
        if self.fail_on is not None and any(int(v.flat[0]) == self.fail_on for v in volumes):
            raise RuntimeError("planted failure")
        return [("result", int(v.flat[0])) for v in volumes]

    def stats(self, device):
        with self.lock:
            kept, peak = self.last.get(threading.get_ident(), (0, 0))
        return {"context_cached_bytes": kept, "context_peak_bytes": peak, "ms_total": self.seconds * 1e3}

    def trim(self, device):
        with self.lock:
            self.kept[threading.get_ident()] = 0
            self.trims += 1


@pytest.fixture
def fake(monkeypatch):
    f = FakeBatch()
    monkeypatch.setattr(serving, "skeletonize_batch", f)
    monkeypatch.setattr(serving, "context_stats", f.stats)
    monkeypatch.setattr(serving, "trim_context", f.trim)
    return f


def volume(tag, edge=16, dtype=np.uint32):
    v = np.zeros((edge, edge, edge), dtype)
    v.flat[0] = tag
    return v


def test_footprint_counts_labels_and_state():
    fixed = serving.REQUEST_BYTES
    assert serving.footprint((10, 10, 10), np.uint64) == 1000 * (8 + serving.STATE_BYTES_PER_VOXEL) + fixed
    assert serving.footprint((10, 10, 10), np.uint8) == 1000 * (1 + serving.STATE_BYTES_PER_VOXEL) + fixed
    assert serving.footprint((10, 10, 10), np.uint8, 300) == 1000 * 301 + fixed


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


def test_kept_blocks_count_against_the_cap_and_are_handed_back(fake):
    fake.keeps = True
    fake.seconds = 0.02
    per = serving.footprint((16, 16, 16), np.uint32)
    with serving.Server(workers=2, memory_cap=2 * per, max_batch=2) as server:
        server.submit(volume(1)).result(timeout=30)  # one worker now keeps one request's blocks
        futures = [server.submit(volume(i)) for i in range(2, 12)]
        for f in futures:
            f.result(timeout=30)
    # what the workers kept plus what ran never passed the cap, and kept blocks were handed back
    assert fake.peak <= 2 * per
    assert server.trims >= 1 and fake.trims == server.trims
    assert len(server.records) == len(server.batches)
    assert sum(r["requests"] for r in server.records) == 11


def test_measured_peaks_raise_the_estimate(fake):
    fake.state = 300
    fake.seconds = 0.0
    edge = 1 + int(round(serving.MEASURE_VOXELS ** (1 / 3)))
    with serving.Server(workers=1) as server:
        server.submit(volume(1, edge=edge, dtype=np.uint8)).result(timeout=30)
        assert server.state_bytes_per_voxel >= 300
        later = server.submit(volume(2))
        later.result(timeout=30)
    assert later.request.bytes == serving.footprint((16, 16, 16), np.uint32, server.state_bytes_per_voxel)
    with serving.Server(workers=1) as server:  # small batches teach nothing
        server.submit(volume(1)).result(timeout=30)
    assert server.state_bytes_per_voxel == serving.STATE_BYTES_PER_VOXEL


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
