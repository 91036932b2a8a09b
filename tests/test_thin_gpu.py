"""GPU parity of the thinning kernels against the oracle (bit-exact).

Every call goes through libbgt.so's C ABI (ctypes).  The oracle is the CPU
restatement in oracle/ (itself pinned against the reference's own code in
tests/test_oracle.py)."""
import numpy as np
import pytest

from oracle import pyoracle as po
from tests.helpers import blobs2d, blobs3d, random2d, random3d

pytestmark = pytest.mark.gpu


def _cases2d(seed=0):
    rng = np.random.default_rng(seed)
    cases = [
        np.zeros((1, 1), np.uint8), np.ones((1, 1), np.uint8), np.ones((3, 3), np.uint8),
        np.zeros((40, 70), np.uint8), np.ones((1, 100), np.uint8), np.ones((100, 1), np.uint8),
        np.ones((17, 33), np.uint8), np.ones((64, 64), np.uint8),
    ]
    for h, w in [(5, 5), (31, 33), (64, 96), (97, 131), (200, 300), (130, 1030)]:
        cases.append(random2d(rng, h, w, 0.5))
        cases.append(random2d(rng, h, w, 0.9))
        cases.append(blobs2d(rng, h, w, max(1, h * w // 800)))
    return cases


def _cases3d(seed=1):
    rng = np.random.default_rng(seed)
    cases = [np.zeros((1, 1, 1), np.uint8), np.ones((3, 3, 3), np.uint8), np.ones((5, 7, 9), np.uint8)]
    for d, h, w in [(6, 7, 9), (20, 33, 35), (40, 40, 70), (33, 64, 65)]:
        cases.append(random3d(rng, d, h, w, 0.5))
        cases.append(blobs3d(rng, d, h, w, max(1, d * h * w // 3000)))
    return cases


def _run_batch(ctx, imgs, cfg, plain):
    import torch
    from begputhinning_b200 import Batch
    b = Batch(ctx)
    ids = [b.add(im.shape, cfg) for im in imgs]
    b.finalize()
    ins = [torch.from_numpy(im).cuda() for im in imgs]
    outs = [torch.empty_like(t) for t in ins]
    for i, t, o in zip(ids, ins, outs):
        b.set_io(i, t, o)
    b.run(plain=bool(plain), device_loop=plain == "device")
    torch.cuda.synchronize()
    res = [o.cpu().numpy() for o in outs]
    stats = [b.stats(i) for i in ids]
    b.close()
    return res, stats


@pytest.mark.parametrize("plain", [False, True, "device"])
def test_thin2d_all_cfgs(ctx, plain):
    from begputhinning_b200 import cfg_list
    imgs = _cases2d()
    want = [po.thin2d(im)[0] for im in imgs]
    for cfg in cfg_list(2):
        got, stats = _run_batch(ctx, imgs, cfg, plain)
        for k, (g, w) in enumerate(zip(got, want)):
            assert np.array_equal(g, w), f"cfg {cfg} case {k} shape {imgs[k].shape}: {(g != w).sum()} px differ"
        assert all(s["converged"] == 1 for s in stats), (cfg, stats)


@pytest.mark.parametrize("plain", [False, True, "device"])
def test_thin3d_all_cfgs(ctx, plain):
    from begputhinning_b200 import cfg_list
    vols = _cases3d()
    want = [po.thin3d(v)[0] for v in vols]
    for cfg in cfg_list(3):
        got, stats = _run_batch(ctx, vols, cfg, plain)
        for k, (g, w) in enumerate(zip(got, want)):
            assert np.array_equal(g, w), f"cfg {cfg} case {k} shape {vols[k].shape}: {(g != w).sum()} vx differ"
        assert all(s["converged"] == 1 for s in stats), (cfg, stats)


def test_plain_device_loop_matches_host_loop(ctx):
    """The plain path with its pass loop on the device runs the same passes
    as the host-driven loop (same pass counts), and its graph replays: the
    second and third runs start from fresh inputs again."""
    import torch
    from begputhinning_b200 import Batch
    rng = np.random.default_rng(12)
    items = [blobs2d(rng, 300, 420, 40), random2d(rng, 97, 131, 0.5), blobs3d(rng, 30, 40, 50, 5),
             random3d(rng, 20, 33, 35, 0.5), np.zeros((9, 9), np.uint8), blobs2d(rng, 1100, 900, 300)]
    want = [po.thin2d(it)[0] if it.ndim == 2 else po.thin3d(it)[0] for it in items]
    b = Batch(ctx)
    ids = [b.add(it.shape) for it in items]
    b.finalize()
    ins = [torch.from_numpy(it).cuda() for it in items]
    outs = [torch.empty_like(t) for t in ins]
    for i, t, o in zip(ids, ins, outs):
        b.set_io(i, t, o)
    b.run(plain=True)
    host = [b.stats(i) for i in ids]
    for r in range(3):
        for o in outs:
            o.fill_(7)
        b.run(plain=True, device_loop=True)
        for k, (o, w) in enumerate(zip(outs, want)):
            assert np.array_equal(o.cpu().numpy(), w), f"run {r} instance {k}"
        dev = [b.stats(i) for i in ids]
        assert [s["passes"] for s in dev] == [s["passes"] for s in host]
        assert all(s["converged"] == 1 for s in dev)
    b.close()


def test_mixed_batch_engine(ctx):
    """2D and 3D instances of uneven size in one persistent launch, default configs."""
    rng = np.random.default_rng(7)
    items = []
    for i in range(24):
        if i % 3 == 2:
            items.append(blobs3d(rng, *rng.integers(8, 48, 3), 4))
        else:
            h, w = rng.integers(16, 400, 2)
            items.append(blobs2d(rng, h, w, max(1, h * w // 1500)))
    got, stats = _run_batch(ctx, items, -1, False)
    for k, (g, it) in enumerate(zip(got, items)):
        w = po.thin2d(it)[0] if it.ndim == 2 else po.thin3d(it)[0]
        assert np.array_equal(g, w), f"instance {k} shape {it.shape}"


def test_engine_repeatable_and_graph(ctx):
    """Replaying the captured graph gives the same result every time."""
    import torch
    from begputhinning_b200 import Batch
    rng = np.random.default_rng(11)
    imgs = [blobs2d(rng, 300, 260, 30), blobs3d(rng, 30, 40, 50, 5)]
    want = [po.thin2d(imgs[0])[0], po.thin3d(imgs[1])[0]]
    b = Batch(ctx)
    ids = [b.add(im.shape) for im in imgs]
    b.finalize()
    ins = [torch.from_numpy(im).cuda() for im in imgs]
    outs = [torch.zeros_like(t) for t in ins]
    for i, t, o in zip(ids, ins, outs):
        b.set_io(i, t, o)
    for rep in range(3):
        for o in outs:
            o.zero_()
        b.run(graph=True)
        torch.cuda.synchronize()
        for o, w in zip(outs, want):
            assert np.array_equal(o.cpu().numpy(), w), f"replay {rep}"
    b.close()


DTYPES = [np.uint8, np.int8, np.uint16, np.int16, np.uint32, np.int32, np.float32, np.float64, np.bool_]


@pytest.mark.parametrize("dt", DTYPES)
def test_thin_dtypes_host_api(ctx, dt):
    """Thinning2D / Thinning3D on every pixel type, with the reference's
    binarisation (2D: (unsigned)v > 0 on the device; 3D: int(v) > 0)."""
    from begputhinning_b200 import Thinning2D, Thinning3D
    from begputhinning_b200.api import dtype_code
    rng = np.random.default_rng(3)
    base = blobs2d(rng, 70, 90, 8)
    vals = np.array([0, 1, 2, -1, 0.5, 1.5, -3.7, 300, 70000], dtype=np.float64)
    noise = rng.integers(0, len(vals), base.shape)
    raw = np.where(base > 0, vals[noise], 0)
    if dt == np.bool_:
        a = raw != 0
    else:
        with np.errstate(all="ignore"):
            a = raw.astype(dt)
    fg = po.binarise(a, dtype_code(a.dtype), 2)
    out = Thinning2D(a, ctx)
    assert out.dtype == a.dtype
    assert np.array_equal(out.astype(np.uint8) != 0, po.thin2d(fg)[0] != 0)
    v3 = np.stack([a] * 6)[:, :40, :50].copy()
    fg3 = po.binarise(v3, dtype_code(v3.dtype), 3)
    out3 = Thinning3D(v3, ctx)
    assert np.array_equal(out3.astype(np.uint8) != 0, po.thin3d(fg3)[0] != 0)


def test_thin_device_api(ctx):
    import torch
    from begputhinning_b200 import thin_device
    rng = np.random.default_rng(5)
    img = blobs2d(rng, 257, 513, 40)
    got = thin_device(torch.from_numpy(img).cuda(), ctx=ctx)
    torch.cuda.synchronize()
    assert np.array_equal(got.cpu().numpy(), po.thin2d(img)[0])


def test_config_shapes_parity(ctx):
    """Generator shapes at reduced size (frame strokes, vessels, trees)."""
    from begputhinning_b200 import Thinning2D, Thinning3D, synth
    img = synth.frame512(0)
    assert np.array_equal(Thinning2D(img, ctx), po.thin2d(img)[0])
    ves = synth.vessels2d(5, 1024, 768, nroots=6)
    assert np.array_equal(Thinning2D(ves, ctx), po.thin2d(ves)[0])
    vol = synth.trees3d(6, 96, 80, 72, ntrees=3, nell=1)
    assert np.array_equal(Thinning3D(vol, ctx), po.thin3d(vol)[0])


@pytest.mark.parametrize("buffers", [1, 2, 3])
def test_pipelined_batch_host_to_host(buffers):
    """Consecutive host-to-host passes through PipelinedBatch (chunks on
    three streams, `buffers` device copies used in turn) give the oracle's
    output on every pass, also when a pass's inputs change between passes."""
    import torch

    from begputhinning_b200 import PipelinedBatch
    rng = np.random.default_rng(40 + buffers)
    shapes = [(24, 30, 40), (64, 96), (97, 131), (1, 1), (40, 70), (130, 200)]
    passes = []
    for p in range(3):
        items = [blobs3d(rng, *s, 3) if len(s) == 3 else random2d(rng, *s, 0.5) for s in shapes]
        passes.append(items)
    pb = PipelinedBatch(shapes, chunks=3, device=0, buffers=buffers)
    total = pb.total
    host_in = [torch.empty(total, dtype=torch.uint8, pin_memory=True) for _ in passes]
    host_out = [torch.zeros(total, dtype=torch.uint8, pin_memory=True) for _ in passes]
    for hin, items in zip(host_in, passes):
        v = hin.numpy()
        for it, o in zip(items, pb.offs):
            v[o:o + it.size] = it.reshape(-1)
    for hin, hout in zip(host_in, host_out):
        pb.run(hin, hout)
    torch.cuda.synchronize()
    for hout, items in zip(host_out, passes):
        v = hout.numpy()
        for it, o in zip(items, pb.offs):
            want = po.thin2d(it)[0] if it.ndim == 2 else po.thin3d(it)[0]
            assert np.array_equal(v[o:o + it.size].reshape(it.shape), want)
    pb.close()


@pytest.mark.parametrize("ctas", [1, 2, 3, 8, 64])
def test_engine_small_grids_and_gangs(ctx, ctas):
    """Volumes and images in one batch on a capped engine grid: with few CTAs
    the gang budget (half the grid) admits only the smallest 3D waves, or
    none, so gangs, ordinary waves and gang-less volumes run side by side;
    every instance must converge to the oracle's result."""
    import torch

    from begputhinning_b200 import Batch
    rng = np.random.default_rng(70 + ctas)
    items = [blobs3d(rng, 20 + 7 * k, 33, 40 + 5 * k, 3) for k in range(4)]
    items += [random3d(rng, 9, 12, 10, 0.5), blobs2d(rng, 97, 131, 10), random2d(rng, 64, 96, 0.5)]
    b = Batch(ctx)
    ids = [b.add(it.shape) for it in items]
    b.set_grid(ctas)
    b.finalize()
    ins = [torch.from_numpy(it).cuda() for it in items]
    outs = [torch.empty_like(t) for t in ins]
    for i, t, o in zip(ids, ins, outs):
        b.set_io(i, t, o)
    for rep in range(2):
        b.run()
        for k, (it, o) in enumerate(zip(items, outs)):
            want = po.thin2d(it)[0] if it.ndim == 2 else po.thin3d(it)[0]
            assert np.array_equal(o.cpu().numpy(), want), f"instance {k}, run {rep}"
            assert b.stats(ids[k])["converged"] == 1
    b.close()


def test_vessels_4096_full_size(ctx):
    """The 4096 x 4096 vessel-tree image (20 roots, branching depth 6, 0.1%
    salt, 50 holes) at full size -- the width at which the reference's own
    Thinning2D divides by zero (2D/LibThinning2D.cu:63-67) -- thinned
    through the host API and as a one-instance batch on the tile rings."""
    from begputhinning_b200 import Thinning2D, synth
    img = synth.vessels4096(1)
    want = po.thin2d(img)[0]
    got = Thinning2D(img, ctx)
    assert np.array_equal(got, want), f"{(got != want).sum()} px differ"
    (ring,), _ = _run_batch(ctx, [img], 2, False)
    assert np.array_equal(ring, want)


def test_benchmark_subset_with_wide_images(ctx):
    """The first 160 images of the benchmark batch's generator -- 26 of them
    1025-2048 pixels wide -- and four tree volumes, thinned together in one
    batch (the wide images are the ones cut into bands)."""
    from begputhinning_b200 import synth
    imgs, vols = synth.mixed_batch(3, 160, 4)
    assert sum(1 for im in imgs if im.shape[1] > 1024) == 26
    items = imgs + vols
    got, stats = _run_batch(ctx, items, -1, False)
    for k, (g, it) in enumerate(zip(got, items)):
        want = po.thin2d(it)[0] if it.ndim == 2 else po.thin3d(it)[0]
        assert np.array_equal(g, want), f"instance {k} shape {it.shape}"
    assert all(s["converged"] == 1 for s in stats)
