"""Parity with the oracle at the benchmark workloads' full sizes, where the engine's scheduling
differs from the small cases (clusters of 4 and 8 CTAs for the large objects, lone-first CTAs, the
page-locked slab-wise input path, wide object counts):

* the 512^3 uint64 dense segmentation (600 Voronoi seeds cut by tubes, seed 1), anisotropy
  (8, 8, 40), from device memory and from page-locked host memory;
* the 64-volume uneven uint32 batch (seed 2), anisotropy (4, 4, 4), through one
  skeletonize_batch call;
* the 1024x1024x256 uint32 dense segmentation (3000 seeds, seed 3), anisotropy (16, 16, 40),
  in-core.

Every skeleton is compared with the oracle's bit for bit (labels, offsets, vertices, edges, radii).
The oracle runs on every host core."""
import os

import numpy as np
import pytest

from oracle import oracle
from test_gpu_parity import CFG0_PARAMS, assert_same, bk

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _device(volume):
    import torch

    return torch.from_numpy(np.ascontiguousarray(volume.transpose(2, 1, 0))).cuda().permute(2, 1, 0)


def test_dense_512_matches_oracle(gpu):
    import torch

    from brook_b200 import synthetic

    volume = synthetic.dense_volume((512, 512, 512), seeds=600, seed=1, dtype=np.uint64)
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(8, 8, 40), dust_threshold=100)
    exp = oracle.skeletonize(volume, threads=THREADS, **opts)
    got = bk().skeletonize(_device(volume), output="packed", **opts)
    assert len(got) > 500
    assert_same(got, exp, "512^3 from device memory")
    pinned_t = torch.empty(volume.shape[::-1], dtype=torch.int64, pin_memory=True)
    pinned_t.numpy().view(np.uint64)[...] = volume.transpose(2, 1, 0)
    pinned = pinned_t.numpy().view(np.uint64).transpose(2, 1, 0)
    assert_same(bk().skeletonize(pinned, output="packed", **opts), exp, "512^3 from page-locked host memory")


def test_uneven_batch_64_matches_oracle(gpu):
    from brook_b200 import synthetic

    volumes = synthetic.uneven_batch(seed=2)
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(4, 4, 4), dust_threshold=100)
    batch = bk().skeletonize_batch([_device(v) for v in volumes], output="packed", **opts)
    assert len(batch) == 64
    total = 0
    for i, v in enumerate(volumes):
        exp = oracle.skeletonize(v, threads=THREADS, **opts)
        assert_same(batch[i], exp, f"batch sample {i} {v.shape}")
        total += len(batch[i])
    assert total > 1000


def test_dense_1024x1024x256_in_core_matches_oracle(gpu):
    from brook_b200 import synthetic

    volume = synthetic.dense_volume((1024, 1024, 256), seeds=3000, seed=3, dtype=np.uint32)
    opts = dict(teasar_params=CFG0_PARAMS, anisotropy=(16, 16, 40), dust_threshold=100)
    exp = oracle.skeletonize(volume, threads=THREADS, **opts)
    got = bk().skeletonize(_device(volume), output="packed", **opts)
    assert len(got) > 2000
    assert_same(got, exp, "1024x1024x256")
