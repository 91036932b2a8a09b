"""CPU: the oracle restatement pinned against the reference's own code.

* golden vectors produced by the reference's rule functions, ExtractSegmentsV
  and CenterlineExtraction (tests/golden/make_golden.py) -- no reference tree
  needed to run these;
* where oracle/_ref exists (built from the reference tree), exhaustive rule
  equality and random end-to-end comparisons against it.
"""
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from tests.helpers import blobs2d, blobs3d, random2d, random3d

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_ref.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def test_golden_2d(golden):
    for k in range(int(golden["n2"])):
        img = golden[f"d2_{k}_in"]
        thin, _ = po.thin2d(img)
        assert np.array_equal(thin, golden[f"d2_{k}_thin"]), f"thin2d case {k}"
        s = po.segments2d(thin)
        assert np.array_equal(s.start, golden[f"d2_{k}_seg_start"])
        assert np.array_equal(s.is_end, golden[f"d2_{k}_seg_end"])
        assert np.array_equal(s.pts, golden[f"d2_{k}_seg_pts"].reshape(s.pts.shape))
        for ml, sp in [(0, 0), (4, 2)]:
            cl = po.centerline2d(img, ml, sp)
            assert np.array_equal(cl.idx, golden[f"d2_{k}_cl_{ml}_{sp}_idx"])
            assert np.array_equal(cl.x.view(np.uint32), golden[f"d2_{k}_cl_{ml}_{sp}_x"].view(np.uint32))
            assert np.array_equal(cl.y.view(np.uint32), golden[f"d2_{k}_cl_{ml}_{sp}_y"].view(np.uint32))


def test_golden_3d(golden):
    for k in range(int(golden["n3"])):
        vol = golden[f"d3_{k}_in"]
        thin, _ = po.thin3d(vol)
        assert np.array_equal(thin, golden[f"d3_{k}_thin"]), f"thin3d case {k}"
        s = po.segments3d(thin)
        assert np.array_equal(s.start, golden[f"d3_{k}_seg_start"])
        assert np.array_equal(s.is_end, golden[f"d3_{k}_seg_end"])
        assert np.array_equal(s.pts, golden[f"d3_{k}_seg_pts"].reshape(s.pts.shape))
        if f"d3_{k}_cl_idx" in golden:
            cl = po.centerline3d(vol, 3, 2)
            assert np.array_equal(cl.idx, golden[f"d3_{k}_cl_idx"])
            for a, key in [(cl.x, "x"), (cl.y, "y"), (cl.z, "z")]:
                assert np.array_equal(a.view(np.uint32), golden[f"d3_{k}_cl_{key}"].view(np.uint32))


def test_known_answers():
    """Hand-made cases: single pixel, 1-px line, empty, filled rectangle, ring."""
    z = np.zeros((9, 9), np.uint8)
    assert not po.thin2d(z)[0].any()
    p = z.copy()
    p[4, 4] = 1
    assert np.array_equal(po.thin2d(p)[0], p)  # a single pixel survives
    line = np.zeros((9, 12), np.uint8)
    line[4, 2:10] = 1
    assert np.array_equal(po.thin2d(line)[0], line)  # a 1-px line is already thin
    rect = np.zeros((20, 30), np.uint8)
    rect[5:15, 4:26] = 1
    t = po.thin2d(rect)[0]
    assert t.sum() > 0 and t.sum() < rect.sum() and (t <= rect).all()
    ring = np.zeros((14, 14), np.uint8)
    ring[3:11, 3:11] = 1
    ring[5:9, 5:9] = 0
    tr = po.thin2d(ring)[0]
    # the hole survives: thinning preserves topology
    assert tr[5:9, 5:9].sum() == 0 and tr.sum() > 0
    segs = po.segments2d(p).as_lists()
    assert segs == [(1, ((4, 4),))]  # isolated point: one single-point end segment
    v = np.zeros((7, 7, 7), np.uint8)
    v[3, 3, 3] = 1
    assert np.array_equal(po.thin3d(v)[0], v)


have_ref = pytest.mark.skipif(not (po.have_ref("2d") and po.have_ref("3d")),
                              reason="oracle/_ref (built from the reference tree) not present")


@have_ref
def test_rule2d_exhaustive_vs_reference():
    """All 2^9 neighbourhoods, four directions: restated rule == reference function."""
    ref = po.ref("2d")
    for d in range(4):
        for cfg in range(512):
            # centre and 8 neighbours; build a 32-bit window where pixel bit 1 is the centre
            c, nbrs = cfg & 1, [(cfg >> (1 + i)) & 1 for i in range(8)]  # N,NE,E,SE,S,SW,W,NW
            up = (nbrs[7] << 0) | (nbrs[0] << 1) | (nbrs[1] << 2)
            cp = (nbrs[6] << 0) | (c << 1) | (nbrs[2] << 2)
            dn = (nbrs[5] << 0) | (nbrs[4] << 1) | (nbrs[3] << 2)
            r = ref.ref2d_rule(d, up, dn, cp)
            ref_del = c & ~((r >> 1) & 1) & 1
            mine = int(po.rule2d(d, np.array([n for n in nbrs], np.uint64))) & c
            assert mine == ref_del, (d, cfg)


@have_ref
@pytest.mark.parametrize("direction", range(6))
def test_rule3d_exhaustive_vs_reference(direction):
    """All 2^26 neighbourhoods of a foreground voxel, per direction."""
    assert po.rule3d_exhaustive_vs_ref(direction) == 0


@have_ref
def test_random_images_vs_reference():
    rng = np.random.default_rng(5)
    for k in range(12):
        h, w = rng.integers(5, 80, 2)
        img = random2d(rng, h, w, rng.random()) if k % 2 else blobs2d(rng, h, w, 5)
        t = po.thin2d(img)[0]
        assert np.array_equal(t, po.ref_thin2d(img))
        assert po.segments2d(t).as_lists() == po.ref_segments2d(t).as_lists()
    for k in range(4):
        d, h, w = rng.integers(5, 22, 3)
        vol = random3d(rng, d, h, w, rng.random()) if k % 2 else blobs3d(rng, d, h, w, 3)
        t = po.thin3d(vol)[0]
        assert np.array_equal(t, po.ref_thin3d(vol))
        assert po.segments3d(t).as_lists() == po.ref_segments3d(t).as_lists()


def test_binarise_rules():
    """Reference binarisation per pixel type (2D on the device, 3D on the host)."""
    f = np.array([0, 0.5, 1.0, -1.0, 3e9, np.nan], np.float32)
    assert po.binarise(f, 7, 2).tolist() == [0, 0, 1, 0, 1, 0]
    assert po.binarise(f, 7, 3).tolist() == [0, 0, 1, 0, 0, 0]
    i8 = np.array([0, 1, -1, 127, -128], np.int8)
    assert po.binarise(i8, 1, 2).tolist() == [0, 1, 1, 1, 1]
    assert po.binarise(i8, 1, 3).tolist() == [0, 1, 0, 1, 0]
    u32 = np.array([0, 1, 2**31, 2**32 - 1], np.uint32)
    assert po.binarise(u32, 5, 2).tolist() == [0, 1, 1, 1]
    assert po.binarise(u32, 5, 3).tolist() == [0, 1, 0, 0]
