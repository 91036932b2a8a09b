"""Generate the golden vectors in tests/golden/ from the reference's own code.

Runs only where the reference tree is present (it loads oracle/_ref, built by
``make -C oracle ref REF=<reference tree>`` from the reference sources: the reference's rule
functions run by a global synchronous host driver, its ExtractSegmentsV and
its CenterlineExtraction).  Inputs are seeded and stored with the outputs, so
the tests need neither the generator nor the reference.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pyoracle as po  # noqa: E402
from tests.helpers import blobs2d, blobs3d, random2d, random3d  # noqa: E402


def segs_arrays(s):
    return s.start.astype(np.int32), s.is_end.astype(np.uint8), s.pts.astype(np.int16)


def main():
    po.build(ref=True)
    assert po.have_ref("2d") and po.have_ref("3d"), "oracle/_ref not built"
    rng = np.random.default_rng(20261203)
    out = {}
    # 2D: thinning + segments of the thinned image + centreline with several parameters
    cases2 = []
    for h, w in [(16, 16), (40, 70), (64, 64), (97, 131), (128, 200)]:
        cases2.append(random2d(rng, h, w, 0.55))
        cases2.append(blobs2d(rng, h, w, max(1, h * w // 700)))
    for k, img in enumerate(cases2):
        thin = po.ref_thin2d(img)
        st, ie, pts = segs_arrays(po.ref_segments2d(thin))
        out[f"d2_{k}_in"] = img
        out[f"d2_{k}_thin"] = thin
        out[f"d2_{k}_seg_start"], out[f"d2_{k}_seg_end"], out[f"d2_{k}_seg_pts"] = st, ie, pts
        for ml, sp in [(0, 0), (4, 2)]:
            cl = po.ref_centerline2d(img.astype(np.uint8), 0, ml, sp)
            out[f"d2_{k}_cl_{ml}_{sp}_x"], out[f"d2_{k}_cl_{ml}_{sp}_y"] = cl.x, cl.y
            out[f"d2_{k}_cl_{ml}_{sp}_idx"] = cl.idx
    # 3D (multiples of 32 for the centreline: the reference pads with
    # uninitialised memory otherwise)
    cases3 = []
    for d, h, w in [(8, 10, 12), (20, 24, 28), (32, 32, 32)]:
        cases3.append(random3d(rng, d, h, w, 0.5))
        cases3.append(blobs3d(rng, d, h, w, 4))
    for k, vol in enumerate(cases3):
        thin = po.ref_thin3d(vol)
        st, ie, pts = segs_arrays(po.ref_segments3d(thin))
        out[f"d3_{k}_in"] = vol
        out[f"d3_{k}_thin"] = thin
        out[f"d3_{k}_seg_start"], out[f"d3_{k}_seg_end"], out[f"d3_{k}_seg_pts"] = st, ie, pts
        if vol.shape == (32, 32, 32):
            cl = po.ref_centerline3d(vol, 0, 3, 2)
            out[f"d3_{k}_cl_x"], out[f"d3_{k}_cl_y"], out[f"d3_{k}_cl_z"] = cl.x, cl.y, cl.z
            out[f"d3_{k}_cl_idx"] = cl.idx
    out["n2"] = np.array(len(cases2))
    out["n3"] = np.array(len(cases3))
    path = os.path.join(HERE, "golden_ref.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
