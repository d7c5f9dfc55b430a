"""A request loop for skeletonization on one GPU with continuous batching.

Requests (label volumes of any size and integer type) arrive at any time through `submit`. A
request is admitted when the device memory it needs (`footprint`) fits under the loop's memory
cap beside what the other workers hold. Each of `workers` threads (one library context, so one
pair of CUDA streams, each) takes every admitted request that is waiting when it becomes free and
runs them as one batch (`skeletonize_batch`: one launch of each engine kernel for all their
objects); a request that arrives while batches are on the GPU joins the next batch a worker
starts, so batches overlap on the device and no request waits for a whole queue to drain.

Memory accounting. A worker holds, while it runs a batch, the batch's footprint plus the blocks
its context kept for reuse from earlier calls; while it is idle, only those kept blocks (read
from the context after every batch). A worker whose batch would not fit beside its own kept
blocks hands them back to the driver first; a worker that cannot admit the oldest waiting request
because of what the idle workers keep asks them to hand theirs back. The per-voxel state estimate
starts at STATE_BYTES_PER_VOXEL and rises to what the contexts report as their peak for every
batch of at least MEASURE_VOXELS voxels (never falls).

A request's result does not depend on the batch it ran in: every volume keeps its own arena, and
the engine's result for an object depends only on that object's voxels.
"""
from __future__ import annotations

import collections
import math
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from .batch import skeletonize_batch

# Device bytes per voxel beyond the labels: component ids, neighbour masks, DBF, the per-voxel
# engine state (PDRF, distances, DAF, flags, liveness, claim keys), union-find / scan scratch, the
# EDT's envelope stacks, the per-object worklists and the allocator's size-class rounding. The
# context's high-water marks measured 157 bytes per voxel for a 512^3 dense volume (22 % of it
# foreground) and 142 for nine overlapping 512x512x256 chunks (44 %).
STATE_BYTES_PER_VOXEL = 160
# Device bytes per request that do not scale with its voxels: per-volume tables, the face stack
# of its border targets, size-class rounding of its small buffers.
REQUEST_BYTES = 4 << 20
# Batches from this many voxels on raise the per-voxel estimate to what they measured (smaller
# ones are dominated by the fixed part).
MEASURE_VOXELS = 1 << 22
# Headroom over a measured per-voxel figure.
MEASURE_MARGIN = 1.05


def footprint(shape, dtype, state_bytes_per_voxel=STATE_BYTES_PER_VOXEL) -> int:
    """Device bytes one request holds while it runs."""
    n = int(np.prod(shape))
    return n * (np.dtype(dtype).itemsize + int(state_bytes_per_voxel)) + REQUEST_BYTES


def context_stats(device):
    """The calling thread's context's statistics of its last call (stage times, work counters, and
    its memory: context_cached_bytes kept for reuse, context_peak_bytes the most held at once)."""
    from . import _native

    return _native.stats(device)


def share_engine(device, percent):
    """Sets the share of the GPU's resident clusters the calling thread's context's persistent
    engine launches take (below 100 they leave room for another worker's kernels)."""
    from . import _native

    _native.set_engine_share(percent, device)


def trim_context(device):
    """Hands the calling thread's context's kept blocks back to the driver."""
    from . import _native

    _native.trim(device)


@dataclass
class Request:
    volume: np.ndarray
    arrival: float
    future: Future = field(default_factory=Future)
    bytes: int = 0
    started: float = 0.0
    finished: float = 0.0

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class Server:
    """Continuous-batching skeletonization server (see the module docstring). `engine_share`
    (percent of the GPU's resident clusters) lets each worker's persistent engine launches leave
    room for the other workers' kernels.

    `submit(volume)` returns a Future whose result is the request's PackedSkeletons; the
    Request object (arrival, start and finish times) is available as `future.request`."""

    def __init__(self, teasar_params=None, anisotropy=(1, 1, 1), dust_threshold=1000, fix_branching=True,
                 fix_borders=True, memory_cap=80e9, workers=2, max_batch=64, device=0, engine_share=100):
        from . import DEFAULT_TEASAR_PARAMS

        self.options = dict(teasar_params=DEFAULT_TEASAR_PARAMS if teasar_params is None else teasar_params,
                            anisotropy=anisotropy, dust_threshold=dust_threshold, fix_branching=fix_branching,
                            fix_borders=fix_borders, device=device)
        self.device = device
        self.engine_share = int(engine_share)
        self.memory_cap = int(memory_cap)
        self.max_batch = int(max_batch)
        self.state_bytes_per_voxel = STATE_BYTES_PER_VOXEL
        self._waiting: collections.deque[Request] = collections.deque()
        n = int(workers)
        self._kept = [0] * n      # blocks each worker's context keeps for reuse
        self._running = [0] * n   # footprint of each worker's running batch
        self._trim_wanted = False
        self._cond = threading.Condition()
        self._closed = False
        self.batches: list[int] = []  # size of every batch run, in start order
        self.records: list[dict] = []  # per batch run: wall times, size and the library's stage times
        self.trims = 0                # hand-backs of kept blocks
        self._threads = [threading.Thread(target=self._work, args=(i,), name=f"brook-b200-worker-{i}", daemon=True)
                         for i in range(n)]
        for t in self._threads:
            t.start()

    def held(self) -> int:
        """Device bytes the workers hold now (running batches and kept blocks)."""
        with self._cond:
            return sum(self._kept) + sum(self._running)

    def submit(self, volume, arrival=None) -> Future:
        volume = np.asarray(volume)
        req = Request(volume, time.perf_counter() if arrival is None else arrival)
        req.bytes = footprint(volume.shape, volume.dtype, self.state_bytes_per_voxel)
        if req.bytes > self.memory_cap:
            raise ValueError(f"brook_b200: a request of {req.bytes} device bytes exceeds the memory cap")
        req.future.request = req
        with self._cond:
            if self._closed:
                raise RuntimeError("brook_b200: the server is closed")
            self._waiting.append(req)
            self._cond.notify()
        return req.future

    def _admit(self, w):
        """Under the lock: the waiting requests (oldest first) that fit beside what the other
        workers hold, with this worker's own kept blocks handed back if need be."""
        others = sum(self._kept[i] + self._running[i] for i in range(len(self._kept)) if i != w)
        budget = self.memory_cap - others
        batch, need = [], 0
        while self._waiting and len(batch) < self.max_batch:
            req = self._waiting[0]
            req.bytes = footprint(req.volume.shape, req.volume.dtype, self.state_bytes_per_voxel)
            if req.bytes > self.memory_cap:  # the estimate rose after it was submitted
                self._waiting.popleft()
                req.future.set_exception(ValueError(
                    f"brook_b200: a request of {req.bytes} device bytes exceeds the memory cap"))
                continue
            if need + req.bytes > budget:
                break
            self._waiting.popleft()
            need += req.bytes
            batch.append(req)
        if not batch and self._waiting and any(self._kept[i] for i in range(len(self._kept)) if i != w):
            self._trim_wanted = True  # the idle workers' kept blocks are in the way
            self._cond.notify_all()
        return batch, need, budget

    def _work(self, w):
        if self.engine_share != 100:
            try:
                share_engine(self.device, self.engine_share)
            except Exception:  # no device: the batches will say so
                pass
        while True:
            with self._cond:
                while True:
                    if self._trim_wanted and self._kept[w]:
                        action = "hand back"
                        break
                    batch, need, budget = self._admit(w)
                    if batch:
                        action = "run"
                        self._trim_wanted = False
                        trim_first = self._kept[w] + need > budget
                        self._running[w] = need
                        self.batches.append(len(batch))
                        break
                    if self._closed and not self._waiting:
                        return
                    self._cond.wait()
            if action == "hand back":
                self._hand_back(w)
                continue
            if trim_first:
                self._hand_back(w)
            start = time.perf_counter()
            try:
                result = skeletonize_batch([r.volume for r in batch], output="packed", **self.options)
                error = None
            except Exception as e:  # every request of the batch reports the failure
                result, error = None, e
            done = time.perf_counter()
            st = self._stats()
            kept, peak = int(st.get("context_cached_bytes", 0)), int(st.get("context_peak_bytes", 0))
            voxels = sum(int(r.volume.size) for r in batch)
            record = {"worker": w, "start": start, "end": done, "requests": len(batch), "voxels": voxels,
                      "handed_back_first": trim_first, "failed": error is not None,
                      "device_ms": st.get("ms_total"), "kept_bytes": kept, "peak_bytes": peak,
                      "host_ms": {k[8:]: v for k, v in st.items() if k.startswith("host_ms_")}}
            with self._cond:
                self.records.append(record)
                self._running[w] = 0
                self._kept[w] = kept
                if error is None and voxels >= MEASURE_VOXELS and peak:
                    labels = sum(int(r.volume.nbytes) for r in batch)
                    per = (peak - labels - REQUEST_BYTES * len(batch)) / voxels
                    self.state_bytes_per_voxel = max(self.state_bytes_per_voxel, math.ceil(per * MEASURE_MARGIN))
                self._cond.notify_all()
            for i, r in enumerate(batch):
                r.started, r.finished = start, done
                if error is not None:
                    r.future.set_exception(error)
                else:
                    r.future.set_result(result[i])

    def _stats(self):
        try:
            return context_stats(self.device)
        except Exception:  # no reading: count nothing kept, learn nothing
            return {}

    def _hand_back(self, w):
        trim_context(self.device)
        with self._cond:
            self._kept[w] = 0
            self.trims += 1
            self._cond.notify_all()

    def close(self, wait=True):
        with self._cond:
            self._closed = True
            self._cond.notify_all()
        if wait:
            for t in self._threads:
                t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def replay(requests, server_factory, time_scale=1.0):
    """Submits (arrival, volume) pairs at their arrival times (seconds from now, scaled) and waits
    for every result; returns the Request objects in submission order."""
    futures = []
    with server_factory() as server:
        t0 = time.perf_counter()
        for arrival, volume in requests:
            due = t0 + arrival * time_scale
            now = time.perf_counter()
            if due > now:
                time.sleep(due - now)
            futures.append(server.submit(volume, arrival=due))  # a late submission still counts from `due`
        for f in futures:
            f.exception()
    return [f.request for f in futures]


def percentiles(latencies, qs=(50, 99)):
    a = np.asarray(latencies, np.float64)
    return {f"p{q}": float(np.percentile(a, q)) for q in qs} if a.size else {f"p{q}": None for q in qs}


__all__ = ["Server", "Request", "footprint", "replay", "percentiles", "STATE_BYTES_PER_VOXEL", "REQUEST_BYTES"]
