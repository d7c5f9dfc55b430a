"""Batches split over ranks (brook_b200.sharding): the partition, and a world-size-2 run over the
gloo backend on CPU with a stand-in for the per-rank skeletonize_batch (the real one needs a GPU),
checking that every volume is done once and the gathered result is in the batch's order."""
import os
import socket

import numpy as np
import pytest

from brook_b200 import sharding


def test_partition_is_longest_first_to_the_least_loaded():
    work = [5, 100, 7, 60, 40, 3]
    shares = sharding.partition(work, 2)
    assert sorted(i for s in shares for i in s) == list(range(6))
    loads = [sum(work[i] for i in s) for s in shares]
    assert shares == [[1, 2], [0, 3, 4, 5]]  # 100 | 60 + 40; tie at 100: 7 to rank 0; 5 and 3 to rank 1
    assert max(loads) - min(loads) <= max(work)


def test_partition_single_rank_and_more_ranks_than_units():
    assert sharding.partition([3, 1, 2], 1) == [[0, 1, 2]]
    shares = sharding.partition([3, 1], 4)
    assert sorted(len(s) for s in shares) == [0, 0, 1, 1]
    with pytest.raises(ValueError):
        sharding.partition([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_batch(samples, output, **options):
    from brook_b200 import PackedSkeletons
    from brook_b200.batch import BatchedSkeletons

    parts = []
    for v in samples:
        tag = int(np.asarray(v).flat[0])
        parts.append(PackedSkeletons(np.array([tag], np.int64), np.array([0, 2], np.int64), np.array([0, 1], np.int64),
                                     np.full((2, 3), tag, np.float32), np.array([[0, 1]], np.uint32),
                                     np.ones(2, np.float32), (1.0, 1.0, 1.0)))
    return BatchedSkeletons.concatenate(parts, (1, 1, 1))


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    from brook_b200 import batch

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    done = []

    def recording(samples, output, **options):
        done.extend(int(np.asarray(v).flat[0]) for v in samples)
        return _fake_batch(samples, output, **options)

    batch.skeletonize_batch = recording
    samples = [np.full(shape, tag, np.uint32) for tag, shape in
               [(11, (4, 4, 4)), (12, (9, 9, 9)), (13, (2, 2, 2)), (14, (7, 7, 7)), (15, (5, 5, 5))]]
    result = sharding.skeletonize_batch_sharded(samples, anisotropy=(1, 1, 1))
    np.save(os.path.join(out_dir, f"done{rank}.npy"), np.asarray(done))
    if rank == 0:
        np.save(os.path.join(out_dir, "labels.npy"), np.asarray(result.labels))
        np.save(os.path.join(out_dir, "sample.npy"), np.asarray(result.sample))
    else:
        assert result is None
    dist.destroy_process_group()


def test_two_ranks_over_gloo_gather_in_batch_order(tmp_path):
    import torch.multiprocessing as mp

    mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    done = [np.load(tmp_path / f"done{r}.npy").tolist() for r in range(2)]
    assert sorted(done[0] + done[1]) == [11, 12, 13, 14, 15]  # every volume exactly once
    assert set(done[0]).isdisjoint(done[1])
    assert np.load(tmp_path / "labels.npy").tolist() == [11, 12, 13, 14, 15]
    assert np.load(tmp_path / "sample.npy").tolist() == [0, 1, 2, 3, 4]


def test_iter_chunks_tiles_with_overlap():
    chunks = list(sharding.iter_chunks((1024, 1024, 256), (512, 512, 256), overlap=64))
    assert len(chunks) == 9
    assert chunks[0] == (slice(0, 512), slice(0, 512), slice(0, 256))
    assert chunks[-1] == (slice(896, 1024), slice(896, 1024), slice(0, 256))
    covered = np.zeros((1024, 1024), bool)
    for c in chunks:
        covered[c[0], c[1]] = True
    assert covered.all()
