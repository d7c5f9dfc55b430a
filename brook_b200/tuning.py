"""The object engine's launch choices, measured: `autotune` times candidate choices on the
caller's own volumes (the C ABI's brook_autotune: a coordinate search over the cluster width, the
cluster thresholds and the lone-first share, the engine's device time per candidate), installs the
fastest for the volumes' workload class in the calling thread's context, and saves it in a JSON
table keyed by GPU name and workload class. Every context made later loads the table's entries for
its GPU, so a tuned class stays tuned across processes.

The table lives at $BROOK_B200_TUNING_CACHE, else ~/.cache/brook_b200/tuning.json."""
from __future__ import annotations

import ctypes
import json
import os
import threading

import numpy as np

from . import _native

_lock = threading.Lock()
FIELDS = ("trace_cluster_ctas", "trace_cluster_voxels", "prepare_cluster_voxels", "lone_first_percent")


def cache_path():
    return os.environ.get("BROOK_B200_TUNING_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "brook_b200",
                                                                     "tuning.json")


def _gpu_name(device):
    try:
        import torch

        return torch.cuda.get_device_name(device)
    except Exception:  # pragma: no cover
        return f"device{device}"


def _read():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def install_saved(context, device):
    """Installs the saved choices for this GPU into a new context (nothing when there are none)."""
    table = _read().get(_gpu_name(device), {})
    for key, entry in table.items():
        t = _native.Tuning(*(int(entry[f]) for f in FIELDS))
        _native.check(_native.load().brook_context_set_tuning(context, int(key, 16), ctypes.byref(t)))


def autotune(samples, teasar_params=None, anisotropy=(1, 1, 1), dust_threshold=1000, fix_branching=True,
             fix_borders=True, device=0, save=True):
    """Measures launch choices on `samples` (one volume or a list: a batch), installs the fastest for
    their workload class and, with save, records it in the table. Returns
    {"workload_class", "tuning", "engine_ms"}."""
    from ._intake import DEFAULT_TEASAR_PARAMS, _is_device, device_volume, format_labels, teasar

    if not isinstance(samples, (list, tuple)):
        samples = [samples]
    params = teasar(DEFAULT_TEASAR_PARAMS if teasar_params is None else teasar_params)
    anisotropy = tuple(float(a) for a in np.asarray(anisotropy, dtype=np.float32))
    volumes, keep = [], []
    for s in samples:
        if _is_device(s):
            v, k = device_volume(s)
        else:
            k = format_labels(s)
            v = _native.host_volume(k)
        volumes.append(v)
        keep.append(k)
    opts = _native.options(params, anisotropy, dust_threshold, fix_branching, fix_borders)
    arr = (_native.Volume * max(len(volumes), 1))(*volumes)
    cls, best, ms = ctypes.c_uint64(), _native.Tuning(), ctypes.c_double()
    ctx = _native.context(device)
    _native.check(_native.load().brook_autotune(ctx, arr, len(volumes), ctypes.byref(opts), ctypes.byref(cls),
                                                ctypes.byref(best), ctypes.byref(ms)))
    entry = {f: int(getattr(best, f)) for f in FIELDS}
    if save:
        with _lock:
            table = _read()
            table.setdefault(_gpu_name(device), {})[f"{cls.value:x}"] = entry
            path = cache_path()
            os.makedirs(os.path.dirname(path), exist_ok=True)
            tmp = path + f".{os.getpid()}.tmp"
            with open(tmp, "w") as f:
                json.dump(table, f, indent=1, sort_keys=True)
            os.replace(tmp, path)
    return {"workload_class": f"{cls.value:x}", "tuning": entry, "engine_ms": ms.value}


__all__ = ["autotune", "install_saved", "cache_path"]
