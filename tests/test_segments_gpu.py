"""GPU parity of device segment extraction and of the whole
CenterlineExtraction path against the oracle: identical segment lists in
the reference's emission order, bit-identical float outputs."""
import numpy as np
import pytest

from oracle import pyoracle as po
from tests.helpers import blobs2d, blobs3d, canonical, random2d, random3d

pytestmark = pytest.mark.gpu


def _thin_cases2d():
    rng = np.random.default_rng(21)
    out = []
    for h, w, kind in [(3, 3, "r"), (16, 16, "r"), (40, 70, "b"), (64, 64, "r"), (120, 200, "b"),
                       (300, 257, "b"), (90, 90, "r")]:
        img = blobs2d(rng, h, w, max(1, h * w // 600)) if kind == "b" else random2d(rng, h, w, 0.45)
        out.append(po.thin2d(img)[0])
    out.append(np.zeros((10, 10), np.uint8))
    one = np.zeros((5, 5), np.uint8)
    one[2, 2] = 1
    out.append(one)
    ring = np.zeros((12, 12), np.uint8)
    ring[3, 3:9] = ring[8, 3:9] = ring[3:9, 3] = ring[3:9, 8] = 1
    out.append(ring)
    return out


def test_segments2d_device(ctx):
    from begputhinning_b200 import ExtractSegmentsV
    for k, img in enumerate(_thin_cases2d()):
        got = ExtractSegmentsV(img, ctx).as_lists()
        want = po.segments2d(img).as_lists()
        assert got == want, f"case {k}: {len(got)} vs {len(want)} segments"


def test_segments2d_raw_masks(ctx):
    """Unthinned masks exercise dense junction clusters and stalls."""
    from begputhinning_b200 import ExtractSegmentsV
    rng = np.random.default_rng(22)
    for k in range(6):
        img = random2d(rng, 40 + 7 * k, 50 + 5 * k, 0.3 + 0.1 * k)
        got = ExtractSegmentsV(img, ctx).as_lists()
        want = po.segments2d(img).as_lists()
        assert got == want, f"case {k}"
        assert canonical(got) == canonical(want)


def test_segments3d_device(ctx):
    from begputhinning_b200 import ExtractSegmentsV
    rng = np.random.default_rng(23)
    for k, (d, h, w) in enumerate([(5, 5, 5), (12, 20, 24), (30, 30, 40), (24, 33, 47)]):
        vol = blobs3d(rng, d, h, w, 4) if k % 2 else random3d(rng, d, h, w, 0.4)
        th = po.thin3d(vol)[0]
        for v in (th, vol):
            got = ExtractSegmentsV(v, ctx).as_lists()
            want = po.segments3d(v).as_lists()
            assert got == want, f"case {k}"


@pytest.mark.parametrize("params", [(0, 0), (3, 2), (10, 5), (-1, 1), (2, 0)])
def test_centerline2d(ctx, params):
    from begputhinning_b200 import CenterlineExtraction
    ml, sp = params
    rng = np.random.default_rng(31)
    for k, (h, w) in enumerate([(64, 64), (100, 150), (250, 130), (33, 517)]):
        img = blobs2d(rng, h, w, max(2, h * w // 700))
        x, y, idx = CenterlineExtraction(img, ml, sp, ctx)
        ref = po.centerline2d(img, ml, sp)
        assert np.array_equal(idx, ref.idx), f"case {k}"
        assert np.array_equal(x.view(np.uint32), ref.x.view(np.uint32))
        assert np.array_equal(y.view(np.uint32), ref.y.view(np.uint32))


@pytest.mark.parametrize("params", [(0, 0), (3, 2), (6, 4)])
def test_centerline3d(ctx, params):
    from begputhinning_b200 import CenterlineExtraction
    ml, sp = params
    rng = np.random.default_rng(32)
    for k, (d, h, w) in enumerate([(20, 30, 40), (33, 40, 35), (64, 64, 64)]):
        vol = blobs3d(rng, d, h, w, 5)
        x, y, z, idx = CenterlineExtraction(vol, ml, sp, ctx)
        ref = po.centerline3d(vol, ml, sp)
        assert np.array_equal(idx, ref.idx), f"case {k}"
        for a, b in [(x, ref.x), (y, ref.y), (z, ref.z)]:
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_centerline_config0(ctx):
    """The 512x512 stroke frame end to end (thinning + segments + CSR)."""
    from begputhinning_b200 import CenterlineExtraction, synth
    img = synth.frame512(0)
    x, y, idx = CenterlineExtraction(img, 5, 2, ctx)
    ref = po.centerline2d(img, 5, 2)
    assert np.array_equal(idx, ref.idx)
    assert np.array_equal(x.view(np.uint32), ref.x.view(np.uint32))
    assert np.array_equal(y.view(np.uint32), ref.y.view(np.uint32))


def test_segments_pixel_walk_path(ctx, monkeypatch):
    """The per-component pixel walk (the fallback of the node-parallel walk)
    against the oracle, on thinned images, raw masks and volumes."""
    from begputhinning_b200 import ExtractSegmentsV
    monkeypatch.setenv("BGT_SEGMENTS_PIXEL_WALK", "1")
    rng = np.random.default_rng(24)
    cases = _thin_cases2d()[:6] + [random2d(rng, 45, 52, 0.4)]
    for k, img in enumerate(cases):
        assert ExtractSegmentsV(img, ctx).as_lists() == po.segments2d(img).as_lists(), f"case {k}"
    vol = blobs3d(rng, 20, 24, 28, 4)
    for v in (po.thin3d(vol)[0], vol):
        assert ExtractSegmentsV(v, ctx).as_lists() == po.segments3d(v).as_lists()


def test_segments_large_images(ctx):
    """Stroke networks large enough that one component spans the image."""
    from begputhinning_b200 import ExtractSegmentsV, Thinning2D, synth
    for w, n in [(700, 22), (1100, 50)]:
        img = Thinning2D(synth.strokes2d(9, w, w, n))
        assert ExtractSegmentsV(img, ctx).as_lists() == po.segments2d(img).as_lists()
