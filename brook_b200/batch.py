"""`skeletonize_batch`: independent samples of uneven shapes in one call (the reference's
src/brook/batch.py:193-232). Every object of every sample is traced in the same launches of the
object engine, largest objects first; result[i] equals skeletonize(samples[i], ...)."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native
from ._intake import DEFAULT_TEASAR_PARAMS, _is_device, _run, device_volume, format_labels, producer_stream, teasar
from ._packed import PackedSkeletons


@dataclass
class BatchedSkeletons:
    """Every skeleton of every sample, packed in sample order: `labels[k]` is skeleton k's label in
    its own sample, `sample[k]` its sample index and `s_off[i]:s_off[i+1]` the skeleton range of
    sample i. Vertices are in each sample's own frame."""

    packed: PackedSkeletons
    labels: np.ndarray
    sample: np.ndarray
    s_off: np.ndarray

    def __len__(self):
        return int(self.s_off.size) - 1

    @property
    def vertices(self):
        return self.packed.vertices

    @property
    def edges(self):
        return self.packed.edges

    @property
    def radii(self):
        return self.packed.radii

    @property
    def v_off(self):
        return self.packed.v_off

    @property
    def e_off(self):
        return self.packed.e_off

    @property
    def on_device(self):
        return self.packed.on_device

    def __getitem__(self, i):
        i = int(i)
        if i < 0:
            i += len(self)
        if not 0 <= i < len(self):
            raise IndexError(i)
        lo, hi = int(self.s_off[i]), int(self.s_off[i + 1])
        p = self.packed.to_host()
        return PackedSkeletons(self.labels[lo:hi], p.v_off[lo:hi + 1] - p.v_off[lo], p.e_off[lo:hi + 1] - p.e_off[lo],
                               p.vertices[p.v_off[lo]:p.v_off[hi]], p.edges[p.e_off[lo]:p.e_off[hi]],
                               p.radii[p.v_off[lo]:p.v_off[hi]], p.anisotropy)

    def to_host(self):
        return self if not self.on_device else BatchedSkeletons(self.packed.to_host(), self.labels, self.sample, self.s_off)

    def to_skeletons(self):
        """list[dict[label, Skeleton]], one dict per sample."""
        return [self[i].to_skeletons() for i in range(len(self))]

    @classmethod
    def concatenate(cls, parts, anisotropy):
        labels, sample, s_off, voff, eoff = [], [], [0], [0], [0]
        vertices, edges, radii = [], [], []
        for i, p in enumerate(parts):
            labels.append(p.labels)
            sample.append(np.full(len(p), i, np.int64))
            s_off.append(s_off[-1] + len(p))
            voff.extend((voff[-1] + p.v_off[1:]).tolist())
            eoff.extend((eoff[-1] + p.e_off[1:]).tolist())
            vertices.append(p.vertices)
            edges.append(p.edges)
            radii.append(p.radii)
        cat = lambda xs, shape, dtype: np.concatenate(xs).astype(dtype, copy=False) if xs else np.zeros(shape, dtype)
        if parts and parts[0].on_device:  # device arrays stay on the device
            import torch

            def dcat(xs, shape, dtype):
                if not xs:
                    return torch.zeros(shape, dtype=dtype, device="cuda")
                if dtype == torch.uint32:  # concatenated through a same-width signed view
                    return torch.cat([x.view(torch.int32) for x in xs]).view(torch.uint32)
                return torch.cat(xs)

            arrays = (dcat(vertices, (0, 3), torch.float32), dcat(edges, (0, 2), torch.uint32),
                      dcat(radii, (0,), torch.float32))
        else:
            arrays = (cat(vertices, (0, 3), np.float32), cat(edges, (0, 2), np.uint32), cat(radii, (0,), np.float32))
        packed = PackedSkeletons(cat(labels, (0,), np.int64), np.asarray(voff, np.int64), np.asarray(eoff, np.int64),
                                 *arrays, tuple(float(a) for a in anisotropy))
        return cls(packed, packed.labels, cat(sample, (0,), np.int64), np.asarray(s_off, np.int64))


def _is_point(entry):
    """A single 3-D point, rather than one sample's sequence of points."""
    if isinstance(entry, np.ndarray):
        return entry.ndim == 1 and entry.shape[0] == 3
    if entry is None or isinstance(entry, (str, bytes)):
        return False
    try:
        values = list(entry)
    except TypeError:
        return False
    return len(values) == 3 and all(np.ndim(value) == 0 for value in values)


def sample_targets(targets, count, name):
    """One list of (x, y, z) points per sample, in each sample's own frame, with the rules of the
    reference's batch (src/brook/batch.py:173-190): None or an empty sequence means no sample has
    targets; otherwise one entry per sample (None or an empty sequence for a sample without any);
    a flat list of points is refused."""
    if targets is None:
        return None
    entries = list(targets)
    if not entries:
        return None
    if any(_is_point(entry) for entry in entries):
        raise ValueError(f"brook_b200: {name} is per sample in a batch: pass one sequence of points for each sample "
                         f"(an empty sequence for a sample without targets), not one flat list of points")
    if len(entries) != count:
        raise ValueError(f"brook_b200: {name} has {len(entries)} entries for {count} samples")
    return [[] if entry is None else [tuple(int(c) for c in point) for point in entry] for entry in entries]


def skeletonize_batch(samples, teasar_params=DEFAULT_TEASAR_PARAMS, anisotropy=(1, 1, 1), dust_threshold=1000,
                      fix_branching=True, fix_borders=True, fill_holes=False, fix_avocados=False,
                      extra_targets_before=None, extra_targets_after=None, progress=False, output="packed_device",
                      stream=None, borrow=True, voxel_graph=None, device=0):
    """Skeletonize independent samples (host arrays or CUDA arrays; shapes may differ) in one call.

    `extra_targets_before` / `extra_targets_after` are per sample: a sequence aligned with
    `samples` holding each sample's own points (an empty sequence or None for a sample without
    targets). `stream` is the producer's stream that the library waits for before reading device
    samples (default: each array's own CUDA array interface stream, torch's current stream for
    torch tensors, else the legacy default stream). Returns BatchedSkeletons with CUDA tensors
    that the library produced on the device (output="packed_device"), with host arrays
    ("packed"), or a list of {label: Skeleton} dicts ("skeletons")."""
    if output not in ("packed_device", "packed", "skeletons"):
        raise ValueError("brook_b200: output must be 'packed_device', 'packed' or 'skeletons'")
    if voxel_graph is not None:
        raise NotImplementedError("brook_b200: voxel_graph is not supported")
    if isinstance(samples, np.ndarray) and samples.ndim == 4:
        samples = list(samples)
    samples = list(samples)
    before = sample_targets(extra_targets_before, len(samples), "extra_targets_before")
    after = sample_targets(extra_targets_after, len(samples), "extra_targets_after")
    targets = None
    if before is not None or after is not None:
        targets = [(before[i] if before else [], after[i] if after else []) for i in range(len(samples))]
    params = teasar(teasar_params)
    anisotropy = tuple(float(a) for a in np.asarray(anisotropy, dtype=np.float32))
    volumes, keep, producers = [], [], []
    for s in samples:
        if _is_device(s):
            v, k = device_volume(s)
            producers.append(producer_stream(s, stream))
        else:
            k = format_labels(s)
            v = _native.host_volume(k)
        volumes.append(v)
        keep.append(k)
    parts = _run(volumes, params, anisotropy, None, dust_threshold, fix_branching, fix_borders, [], [], device,
                 device_output=output == "packed_device", producers=producers, sample_targets=targets,
                 fill_holes=fill_holes, fix_avocados=fix_avocados) \
        if volumes else []
    result = BatchedSkeletons.concatenate(parts, anisotropy)
    if output == "skeletons":
        return result.to_skeletons()
    if output == "packed_device" and not result.on_device:  # an empty batch
        return BatchedSkeletons(result.packed.to_device(), result.labels, result.sample, result.s_off)
    return result


__all__ = ["skeletonize_batch", "BatchedSkeletons"]
