"""A request loop for skeletonization on one GPU with continuous batching.

Requests (label volumes of any size and integer type) arrive at any time through `submit`. A
request is admitted when the device memory it needs (`footprint`) fits under the loop's memory
cap beside the requests already in flight. Each of `workers` threads (one library context, so one
pair of CUDA streams, each) takes every admitted request that is waiting when it becomes free and
runs them as one batch (`skeletonize_batch`: one launch of each engine kernel for all their
objects); a request that arrives while batches are on the GPU joins the next batch a worker
starts, so batches overlap on the device and no request waits for a whole queue to drain.

A request's result does not depend on the batch it ran in: every volume keeps its own arena, and
the engine's result for an object depends only on that object's voxels.
"""
from __future__ import annotations

import collections
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


def footprint(shape, dtype) -> int:
    """Device bytes one request holds while it runs."""
    n = int(np.prod(shape))
    return n * (np.dtype(dtype).itemsize + STATE_BYTES_PER_VOXEL)


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
    """Continuous-batching skeletonization server (see the module docstring).

    `submit(volume)` returns a Future whose result is the request's PackedSkeletons; the
    Request object (arrival, start and finish times) is available as `future.request`."""

    def __init__(self, teasar_params=None, anisotropy=(1, 1, 1), dust_threshold=1000, fix_branching=True,
                 fix_borders=True, memory_cap=80e9, workers=2, max_batch=64, device=0):
        from . import DEFAULT_TEASAR_PARAMS

        self.options = dict(teasar_params=DEFAULT_TEASAR_PARAMS if teasar_params is None else teasar_params,
                            anisotropy=anisotropy, dust_threshold=dust_threshold, fix_branching=fix_branching,
                            fix_borders=fix_borders, device=device)
        self.memory_cap = int(memory_cap)
        self.max_batch = int(max_batch)
        self._waiting: collections.deque[Request] = collections.deque()
        self._in_flight = 0
        self._cond = threading.Condition()
        self._closed = False
        self.batches: list[int] = []  # size of every batch run, in start order
        self._threads = [threading.Thread(target=self._work, name=f"brook-b200-worker-{i}", daemon=True)
                         for i in range(int(workers))]
        for t in self._threads:
            t.start()

    def submit(self, volume, arrival=None) -> Future:
        volume = np.asarray(volume)
        req = Request(volume, time.perf_counter() if arrival is None else arrival)
        req.bytes = footprint(volume.shape, volume.dtype)
        if req.bytes > self.memory_cap:
            raise ValueError(f"brook_b200: a request of {req.bytes} device bytes exceeds the memory cap")
        req.future.request = req
        with self._cond:
            if self._closed:
                raise RuntimeError("brook_b200: the server is closed")
            self._waiting.append(req)
            self._cond.notify()
        return req.future

    def _admit(self):
        """Under the lock: the waiting requests (oldest first) that fit beside those in flight."""
        batch = []
        while self._waiting and len(batch) < self.max_batch:
            req = self._waiting[0]
            if self._in_flight + req.bytes > self.memory_cap:
                break
            self._waiting.popleft()
            self._in_flight += req.bytes
            batch.append(req)
        return batch

    def _work(self):
        while True:
            with self._cond:
                while True:
                    batch = self._admit()
                    if batch or (self._closed and not self._waiting):
                        break
                    self._cond.wait()
                if not batch:
                    return
                self.batches.append(len(batch))
            start = time.perf_counter()
            try:
                result = skeletonize_batch([r.volume for r in batch], output="packed", **self.options)
                error = None
            except Exception as e:  # every request of the batch reports the failure
                result, error = None, e
            done = time.perf_counter()
            with self._cond:
                self._in_flight -= sum(r.bytes for r in batch)
                self._cond.notify_all()
            for i, r in enumerate(batch):
                r.started, r.finished = start, done
                if error is not None:
                    r.future.set_exception(error)
                else:
                    r.future.set_result(result[i])

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


__all__ = ["Server", "Request", "footprint", "replay", "percentiles", "STATE_BYTES_PER_VOXEL"]
