"""Packed skeletons and the per-object Skeleton, as the reference's brook.PackedSkeletons
(src/brook/_packed.py) and the osteoid.Skeleton it returns for output="skeletons"."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


class Skeleton:
    """One object's skeleton in physical space: vertices (V, 3) float32, edges (E, 2) uint32,
    radii (V,) float32 (the DBF at each vertex); `id` is the object's label. When osteoid is
    installed, ``to_osteoid()`` gives the class Kimimaro returns."""

    def __init__(self, vertices, edges, radii, segid, anisotropy):
        self.vertices = vertices
        self.edges = edges
        self.radii = radii
        self.id = int(segid)
        self.anisotropy = tuple(anisotropy)
        a = anisotropy
        self.transform = np.array([[a[0], 0, 0, 0], [0, a[1], 0, 0], [0, 0, a[2], 0]], np.float32)

    def to_osteoid(self):
        from osteoid import Skeleton as OsteoidSkeleton

        return OsteoidSkeleton(self.vertices, self.edges, radii=self.radii, segid=self.id, space="physical",
                               transform=self.transform.copy())

    def __repr__(self):
        return f"Skeleton(id={self.id}, vertices={len(self.vertices)}, edges={len(self.edges)})"


def torch_int32():
    import torch

    return torch.int32


@dataclass
class PackedSkeletons:
    """Skeletons in flat arrays: skeleton k has label `labels[k]`, vertices
    `vertices[v_off[k]:v_off[k+1]]` (float32, physical units), the same range of `radii`, and edges
    `edges[e_off[k]:e_off[k+1]]` (uint32, local to the skeleton)."""

    labels: np.ndarray
    v_off: np.ndarray
    e_off: np.ndarray
    vertices: object
    edges: object
    radii: object
    anisotropy: tuple

    def __len__(self):
        return int(self.labels.size)

    @property
    def on_device(self):
        return not isinstance(self.vertices, np.ndarray)

    def to_host(self):
        if not self.on_device:
            return self
        edges = self.edges.view(torch_int32()).cpu().numpy().view(np.uint32) if self.edges.numel() else \
            np.zeros((0, 2), np.uint32)
        return type(self)(self.labels, self.v_off, self.e_off, self.vertices.cpu().numpy(), edges,
                          self.radii.cpu().numpy(), self.anisotropy)

    def to_device(self, device=None):
        """The arrays as CUDA tensors (torch) on `device` (default: the current device)."""
        if self.on_device:
            return self
        import torch

        dev = torch.device("cuda" if device is None else device)
        edges = torch.from_numpy(np.ascontiguousarray(self.edges, np.uint32).view(np.int32)).to(dev).view(torch.uint32)
        return type(self)(self.labels, self.v_off, self.e_off, torch.from_numpy(self.vertices).to(dev), edges,
                          torch.from_numpy(self.radii).to(dev), self.anisotropy)

    def to_skeletons(self):
        """{label: Skeleton} in physical space."""
        h = self.to_host()
        out = {}
        for k, label in enumerate(h.labels.tolist()):
            v0, v1 = int(h.v_off[k]), int(h.v_off[k + 1])
            e0, e1 = int(h.e_off[k]), int(h.e_off[k + 1])
            out[int(label)] = Skeleton(h.vertices[v0:v1], h.edges[e0:e1], h.radii[v0:v1], label, self.anisotropy)
        return out

    @classmethod
    def from_arrays(cls, arrays):
        return cls(arrays["labels"], arrays["v_off"], arrays["e_off"], arrays["vertices"], arrays["edges"],
                   arrays["radii"], arrays["anisotropy"])

    @classmethod
    def empty(cls, anisotropy):
        return cls(np.zeros(0, np.int64), np.zeros(1, np.int64), np.zeros(1, np.int64), np.zeros((0, 3), np.float32),
                   np.zeros((0, 2), np.uint32), np.zeros(0, np.float32), tuple(float(a) for a in anisotropy))
