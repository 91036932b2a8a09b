"""GPU parity of the resident kernel (begputhinning_b200/csrc/resident.cu)
against the oracle, bit-exact: single-CTA images, images cut into bands of
CTAs that trade halo rows, sparse-brick volumes, volumes that do not fit and
fall back to the tile rings, and batches forced onto the rings."""
import numpy as np
import pytest

from oracle import pyoracle as po
from tests.helpers import blobs2d, blobs3d, random2d, random3d

pytestmark = pytest.mark.gpu


def _run(ctx, items, rings_only=False, grid=0, runs=1):
    import torch
    from begputhinning_b200 import Batch
    b = Batch(ctx)
    ids = [b.add(it.shape) for it in items]
    if rings_only:
        b.set_engine(True)
    if grid:
        b.set_grid(grid)
    b.finalize()
    plans = [b.plan(i) for i in ids]
    ins = [torch.from_numpy(it).cuda() for it in items]
    outs = [torch.empty_like(t) for t in ins]
    for i, t, o in zip(ids, ins, outs):
        b.set_io(i, t, o)
    res = []
    for _ in range(runs):
        for o in outs:
            o.fill_(7)
        b.run()
        res.append([o.cpu().numpy() for o in outs])
    stats = [b.stats(i) for i in ids]
    b.close()
    return res, plans, stats


def _want(it):
    return po.thin2d(it)[0] if it.ndim == 2 else po.thin3d(it)[0]


def test_resident_images_single_cta(ctx):
    rng = np.random.default_rng(21)
    items = [np.zeros((1, 1), np.uint8), np.ones((3, 3), np.uint8), np.ones((1, 100), np.uint8),
             np.ones((100, 1), np.uint8), np.ones((64, 64), np.uint8)]
    for h, w in [(5, 5), (31, 33), (33, 31), (64, 96), (97, 131), (200, 300), (130, 1030), (70, 2047)]:
        items.append(random2d(rng, h, w, 0.5))
        items.append(blobs2d(rng, h, w, max(1, h * w // 800)))
    # many instances: none is a large share of the batch, so none is cut
    items += [blobs2d(rng, 40, 40, 3) for _ in range(300)]
    (got,), plans, stats = _run(ctx, items)
    for k, (g, it) in enumerate(zip(got, items)):
        assert plans[k][0], f"instance {k} not resident"
        assert np.array_equal(g, _want(it)), f"instance {k} shape {it.shape}: {(g != _want(it)).sum()} px differ"
        assert stats[k]["converged"] == 1


@pytest.mark.parametrize("shape,cut", [((600, 1500), True), ((1500, 600), True), ((2100, 2048), True),
                                       ((333, 70), False), ((97, 4000), True)])
def test_resident_image_bands(ctx, shape, cut):
    """One image per batch: the planner cuts it into bands (at least 32 core
    rows each) that run on separate CTAs and meet after every fourth
    iteration to trade 16 halo rows."""
    rng = np.random.default_rng(sum(shape))
    h, w = shape
    img = blobs2d(rng, h, w, max(1, h * w // 1500), rmax=14)
    (got,), plans, stats = _run(ctx, [img], runs=1)
    assert plans[0][0]
    assert (plans[0][1] > 1) == cut, f"{shape}: plan {plans[0]}"
    assert np.array_equal(got[0], _want(img)), f"{shape}: {(got[0] != _want(img)).sum()} px differ"
    assert stats[0]["converged"] == 1


def test_resident_bands_repeat_and_mix(ctx):
    """Banded images beside single-CTA images and volumes, run twice (the
    band counters and halo buffers start clean on every run)."""
    rng = np.random.default_rng(5)
    items = [blobs2d(rng, 2048, 1900, 2500, rmax=12), blobs2d(rng, 1800, 1200, 1500)]
    items += [blobs2d(rng, *rng.integers(20, 300, 2), 12) for _ in range(20)]
    items += [blobs3d(rng, *rng.integers(10, 60, 3), 5) for _ in range(6)]
    runs, plans, stats = _run(ctx, items, runs=2)
    assert plans[0][1] > 1
    for r, got in enumerate(runs):
        for k, (g, it) in enumerate(zip(got, items)):
            assert np.array_equal(g, _want(it)), f"run {r} instance {k} shape {it.shape}"
    assert all(s["converged"] == 1 for s in stats)


def test_resident_volumes(ctx):
    rng = np.random.default_rng(8)
    items = [np.zeros((1, 1, 1), np.uint8), np.ones((3, 3, 3), np.uint8), np.ones((5, 7, 9), np.uint8),
             np.ones((40, 40, 40), np.uint8)]
    for d, h, w in [(6, 7, 9), (20, 33, 35), (40, 40, 70), (33, 64, 65), (9, 100, 130), (70, 20, 33)]:
        items.append(random3d(rng, d, h, w, 0.5))
        items.append(blobs3d(rng, d, h, w, max(1, d * h * w // 3000)))
    (got,), plans, stats = _run(ctx, items)
    for k, (g, it) in enumerate(zip(got, items)):
        assert plans[k][0]
        assert np.array_equal(g, _want(it)), f"volume {k} shape {it.shape}: {(g != _want(it)).sum()} vx differ"
        assert stats[k]["converged"] == 1


def test_resident_volume_spills_to_rings(ctx):
    """A dense volume with more non-empty bricks than one CTA holds is left
    to the tile rings (flagged on the device), beside volumes that fit."""
    rng = np.random.default_rng(9)
    big = random3d(rng, 64, 200, 200, 0.3)  # 7 x 7 x 16 bricks, all non-empty
    small = blobs3d(rng, 30, 40, 50, 4)
    img = blobs2d(rng, 100, 120, 10)
    (got,), plans, stats = _run(ctx, [big, small, img])
    for k, (g, it) in enumerate(zip(got, [big, small, img])):
        assert np.array_equal(g, _want(it)), f"instance {k}"
        assert stats[k]["converged"] == 1


def test_rings_only_matches(ctx):
    rng = np.random.default_rng(10)
    items = [blobs2d(rng, 300, 260, 30), blobs3d(rng, 30, 40, 50, 5), random2d(rng, 97, 131, 0.5)]
    (got,), plans, _ = _run(ctx, items, rings_only=True)
    assert not any(p[0] for p in plans)
    for g, it in zip(got, items):
        assert np.array_equal(g, _want(it))


@pytest.mark.parametrize("grid", [1, 2, 5])
def test_resident_small_grids(ctx, grid):
    """A capped grid limits the bands an image may be cut into; images that
    need more bands than the grid holds go to the tile rings."""
    rng = np.random.default_rng(30 + grid)
    items = [blobs2d(rng, 2048, 2048, 3000, rmax=12), blobs2d(rng, 500, 700, 200), blobs3d(rng, 30, 50, 60, 6)]
    (got,), plans, _ = _run(ctx, items, grid=grid)
    for p in plans:
        assert p[1] <= grid
    for k, (g, it) in enumerate(zip(got, items)):
        assert np.array_equal(g, _want(it)), f"instance {k} (plan {plans[k]})"


@pytest.mark.parametrize("slab_voxels", ["60000", "300000"])
def test_resident_volume_slabs(ctx, slab_voxels, monkeypatch):
    """Volumes cut into z-slabs of brick layers on separate CTAs, trading two
    halo layers after every iteration (the slab size is lowered so that
    small volumes are cut too)."""
    from begputhinning_b200 import synth
    monkeypatch.setenv("BGT_RES3D_SLAB_VOXELS", slab_voxels)
    rng = np.random.default_rng(int(slab_voxels) % 97)
    items = [blobs3d(rng, 96, 70, 80, 30, rmax=9), synth.trees3d(6, 96, 80, 72, ntrees=3, nell=1),
             random3d(rng, 40, 30, 33, 0.5), blobs3d(rng, 17, 40, 40, 4)]
    runs, plans, stats = _run(ctx, items, runs=2)
    assert plans[0][1] > 1 and plans[1][1] > 1, plans
    for r, got in enumerate(runs):
        for k, (g, it) in enumerate(zip(got, items)):
            assert np.array_equal(g, _want(it)), f"run {r} volume {k} shape {it.shape} plan {plans[k]}"
    assert all(s["converged"] == 1 for s in stats)
