"""fill_holes (holes.cu:38-67; skeletonize.cu:86-90, batch.cu:217-220): every component's voids
(background 6-connected to no face of the component's box) filled before the distance transform,
components in ascending id, a component that an earlier fill painted over is filled no more.

The CPU tests pin the oracle's fill against a restatement of the reference's loop on scipy's
binary_fill_holes (whose default structure is the 6-connected one); the GPU tests check the
CUDA path, which computes every component's voids at once and resolves the order afterwards,
against the oracle: skeletons bit for bit and the filled voxel count."""
import numpy as np
import pytest
from scipy import ndimage

from oracle import oracle

PARAMS = dict(scale=1.5, const=20, pdrf_scale=100000, pdrf_exponent=4)


def hollow_cells(shape=(72, 64, 56), cells=10, seed=0, inner=0.5):
    """Ellipsoidal shells (labels 1..cells) with random wall thickness; about `inner` of their
    cavities hold a ball of another label, some shells overlap."""
    rng = np.random.default_rng(seed)
    v = np.zeros(shape, np.uint32)
    x, y, z = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    for i in range(1, cells + 1):
        r = rng.uniform(5, 13, size=3)
        c = [rng.uniform(r[k] + 1, shape[k] - r[k] - 2) for k in range(3)]
        t = rng.uniform(0.35, 0.6)
        d = ((x - c[0]) / r[0]) ** 2 + ((y - c[1]) / r[1]) ** 2 + ((z - c[2]) / r[2]) ** 2
        v[(d <= 1.0) & (d > t)] = i
        if rng.random() < inner:
            v[d <= t * 0.3] = cells + i
    return v


def nested_shells(shape=(48, 48, 48)):
    """A shell, a smaller shell in its cavity, and a ball in the inner cavity."""
    v = np.zeros(shape, np.uint32)
    x, y, z = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    d = np.sqrt((x - 24) ** 2 + (y - 24) ** 2 + (z - 24) ** 2)
    v[(d <= 20) & (d > 16)] = 5
    v[(d <= 12) & (d > 9)] = 3
    v[d <= 5] = 7
    return v


def long_shell(shape=(1100, 12, 12)):
    """A closed box shell longer than 1024 voxels along x (rows of more than 32 words)."""
    v = np.zeros(shape, np.uint32)
    v[2:1098, 1:11, 1:11] = 4
    v[4:1096, 3:9, 3:9] = 0
    v[500:510, 5:7, 5:7] = 9  # a label in the cavity
    return v


def fill_restated(cc):
    """The reference's loop (holes.cu:38-67) over component ids on scipy's hole filling."""
    ids = cc.copy()
    count = int(ids.max())
    objects = ndimage.find_objects(cc.astype(np.int64))
    disabled = np.zeros(count + 1, bool)
    filled_total = 0
    for i in range(1, count + 1):
        box = objects[i - 1]
        if box is None or disabled[i]:
            continue
        crop = ids[box] == i
        filled = ndimage.binary_fill_holes(crop)
        holes = int((filled & ~crop).sum())
        if not holes:
            continue
        filled_total += holes
        previous = ids[box][filled]
        for p in np.unique(previous):
            if p and p != i:
                disabled[p] = True
        view = ids[box]
        view[filled] = i
    return ids, filled_total


@pytest.mark.parametrize("make", [lambda: hollow_cells(seed=0), lambda: hollow_cells(seed=1, cells=14),
                                  nested_shells])
def test_oracle_fill_matches_the_restated_loop(make):
    labels = make()
    opts = dict(teasar_params=PARAMS, anisotropy=(4, 4, 10), dust_threshold=0)
    plain = oracle.skeletonize(labels, stages=True, threads=8, **opts)
    filled = oracle.skeletonize(labels, stages=True, threads=8, fill_holes=True, **opts)
    expect, total = fill_restated(plain.field("cc"))
    np.testing.assert_array_equal(filled.field("cc"), expect)
    assert int(filled.array("filled")[0]) == total > 0


def test_oracle_fill_of_nested_shells():
    """The outer shell (the lower id) fills its whole cavity, the inner shell and ball included:
    both are painted over and disabled, one skeleton remains."""
    labels = nested_shells()
    opts = dict(teasar_params=PARAMS, anisotropy=(1, 1, 1), dust_threshold=0)
    out = oracle.skeletonize(labels, threads=8, fill_holes=True, **opts)
    assert out.array("labels").tolist() == [5]
    assert len(oracle.skeletonize(labels, threads=8, **opts).array("labels")) == 3


# ---- the CUDA path against the oracle ------------------------------------------------------------


def _gpu_and_oracle(labels, **opts):
    import brook_b200
    from brook_b200 import _native

    got = brook_b200.skeletonize(labels, output="packed", fill_holes=True, **opts)
    stats = _native.stats()
    exp = oracle.skeletonize(labels, threads=8, fill_holes=True, **opts)
    return got, stats, exp


@pytest.mark.gpu
@pytest.mark.parametrize("seed,cells", [(0, 10), (1, 14), (2, 20)])
def test_fill_holes_matches_oracle(gpu, seed, cells):
    from test_gpu_parity import assert_same

    labels = hollow_cells(seed=seed, cells=cells)
    opts = dict(teasar_params=PARAMS, anisotropy=(4, 4, 10), dust_threshold=0)
    got, stats, exp = _gpu_and_oracle(labels, **opts)
    assert stats["hole_filled_voxels"] == int(exp.array("filled")[0]) > 0
    assert_same(got, exp, f"fill_holes seed {seed}")


@pytest.mark.gpu
@pytest.mark.parametrize("make", [nested_shells, long_shell])
def test_fill_holes_nested_and_long_rows(gpu, make):
    from test_gpu_parity import assert_same

    labels = make()
    opts = dict(teasar_params=PARAMS, anisotropy=(1, 1, 1), dust_threshold=0)
    got, stats, exp = _gpu_and_oracle(labels, **opts)
    assert stats["hole_filled_voxels"] == int(exp.array("filled")[0]) > 0
    assert_same(got, exp, make.__name__)


@pytest.mark.gpu
def test_fill_holes_in_a_batch_and_on_dense_cells(gpu):
    import brook_b200
    from brook_b200 import synthetic
    from test_gpu_parity import assert_same

    opts = dict(teasar_params=PARAMS, anisotropy=(4, 4, 10), dust_threshold=0)
    samples = [hollow_cells(seed=3), synthetic.dense_volume((96, 80, 64), seeds=20, seed=4, dtype=np.uint32),
               nested_shells()]
    batch = brook_b200.skeletonize_batch(samples, output="packed", fill_holes=True, **opts)
    for i, v in enumerate(samples):
        assert_same(batch[i], oracle.skeletonize(v, threads=8, fill_holes=True, **opts), f"batch sample {i}")
