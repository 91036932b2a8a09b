"""Seeded synthetic inputs of the workload shapes (uint8 {0,1}, empty outer frame).

* ``frame512``   : 512x512, 12 cubic Bezier strokes, radius U[2,6]
* ``vessels4096``: 4096x4096 vessel-like trees (20 roots, binary branching to
  depth 6, branch length U[40,200], child angle +/-U[15,60] deg, radius 10 -> 1.5),
  0.1% salt pixels, 50 elliptical holes of semi-axes U[2,5]
* ``trees256``   : 256^3, 8 tubular trees (depth 5, length U[20,80], radius
  6 -> 1.5) + 3 solid ellipsoids (semi-axes U[10,25], random rotation)
* ``mixed_batch``: 512 images with width log-uniform 64..2048, aspect
  log-uniform 0.5..2, stroke count scaled to area (12 per 512^2), plus 32
  volumes with sides log-uniform 64..192 and tree/ellipsoid counts scaled to
  volume/256^3
* ``FrameStreams``: temporally correlated 1024x1024 frame streams (strokes
  displaced <= 2 px per frame, radius jitter +/-0.5) and tree volumes with
  sides U[128,320] for the serving workload

All generators are deterministic functions of their seed (xoshiro256** in
libbgt_synth.so).  There is no public dataset behind these shapes; the
generators stand in for one.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import synth


def _u8p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def uniform(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, np.float64)
    synth().bgt_synth_uniform(C.c_uint64(seed & (2**64 - 1)), n, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def strokes2d(seed: int, w: int, h: int, n: int, rmin: float = 2.0, rmax: float = 6.0) -> np.ndarray:
    out = np.empty((h, w), np.uint8)
    synth().bgt_synth_strokes2d(C.c_uint64(seed), w, h, n, rmin, rmax, _u8p(out))
    return out


def render_strokes2d(w: int, h: int, ctrl: np.ndarray, radius: np.ndarray) -> np.ndarray:
    ctrl = np.ascontiguousarray(ctrl, np.float64).reshape(-1, 8)
    radius = np.ascontiguousarray(radius, np.float64).reshape(-1)
    out = np.zeros((h, w), np.uint8)
    synth().bgt_synth_render_strokes2d(w, h, len(radius), ctrl.ctypes.data_as(C.POINTER(C.c_double)),
                                       radius.ctypes.data_as(C.POINTER(C.c_double)), _u8p(out))
    return out


def vessels2d(seed: int, w: int = 4096, h: int = 4096, nroots: int = 20, depth: int = 6, lmin: float = 40,
              lmax: float = 200, amin: float = 15, amax: float = 60, r0: float = 10, r1: float = 1.5,
              salt: float = 0.001, nholes: int = 50, hmin: float = 2, hmax: float = 5) -> np.ndarray:
    out = np.empty((h, w), np.uint8)
    synth().bgt_synth_vessels2d(C.c_uint64(seed), w, h, nroots, depth, lmin, lmax, amin, amax, r0, r1, salt,
                                nholes, hmin, hmax, _u8p(out))
    return out


def trees3d(seed: int, w: int, h: int, d: int, ntrees: int = 8, depth: int = 5, lmin: float = 20,
            lmax: float = 80, amin: float = 15, amax: float = 60, r0: float = 6, r1: float = 1.5,
            nell: int = 3, emin: float = 10, emax: float = 25) -> np.ndarray:
    out = np.empty((d, h, w), np.uint8)
    synth().bgt_synth_trees3d(C.c_uint64(seed), w, h, d, ntrees, depth, lmin, lmax, amin, amax, r0, r1, nell,
                              emin, emax, _u8p(out))
    return out


def frame512(seed: int = 0) -> np.ndarray:
    """512x512 image of 12 Bezier strokes (the plain 2D workload)."""
    return strokes2d(seed, 512, 512, 12)


def vessels4096(seed: int = 1) -> np.ndarray:
    """4096x4096 vessel trees with salt and holes."""
    return vessels2d(seed)


def trees256(seed: int = 2) -> np.ndarray:
    """256^3 volume of tubular trees and ellipsoids."""
    return trees3d(seed, 256, 256, 256)


def mixed_batch_shapes(seed: int = 3, n2d: int = 512, n3d: int = 32):
    """Shapes and per-instance generator parameters of the mixed batch."""
    u = uniform(seed, 3 * n2d + 3 * n3d)
    out2, out3 = [], []
    for i in range(n2d):
        w = int(round(math.exp(math.log(64) + (math.log(2048) - math.log(64)) * u[3 * i])))
        w = min(2048, max(64, w))
        a = math.exp(math.log(0.5) + (math.log(2) - math.log(0.5)) * u[3 * i + 1])
        h = min(2048, max(64, int(round(w * a))))
        n = max(1, int(round(12 * w * h / 512 ** 2)))
        out2.append((w, h, n))
    base = 3 * n2d
    for i in range(n3d):
        s = [int(round(math.exp(math.log(64) + (math.log(192) - math.log(64)) * u[base + 3 * i + k])))
             for k in range(3)]
        s = [min(192, max(64, v)) for v in s]
        vol = s[0] * s[1] * s[2] / 256 ** 3
        out3.append((s[0], s[1], s[2], max(1, int(round(8 * vol))), int(round(3 * vol))))
    return out2, out3


def mixed_batch(seed: int = 3, n2d: int = 512, n3d: int = 32):
    """(list of 2D images, list of 3D volumes) of the mixed batch."""
    s2, s3 = mixed_batch_shapes(seed, n2d, n3d)
    imgs = [strokes2d(seed * 1000003 + 17 * i + 1, w, h, n) for i, (w, h, n) in enumerate(s2)]
    vols = [trees3d(seed * 1000003 + 7919 * (i + 1), w, h, d, ntrees=nt, nell=ne)
            for i, (w, h, d, nt, ne) in enumerate(s3)]
    return imgs, vols


class FrameStreams:
    """Temporally correlated 1024x1024 stroke frames for `streams` concurrent
    streams (48 strokes each, the 512^2 density scaled to the frame area).
    Each new frame displaces every control point by at most 2 px and jitters
    each radius by at most 0.5 px (kept within [1.5, 6.5])."""

    def __init__(self, seed: int = 4, streams: int = 16, size: int = 1024, strokes: int = 48):
        self.size = size
        self.seed = seed
        self.frame_no = [0] * streams
        u = uniform(seed, streams * strokes * 9)
        self.ctrl = []
        self.rad = []
        k = 0
        for _ in range(streams):
            c = u[k:k + strokes * 8].reshape(strokes, 8) * size
            k += strokes * 8
            r = 2 + 4 * u[k:k + strokes]
            k += strokes
            self.ctrl.append(c.copy())
            self.rad.append(r.copy())

    def next(self, stream: int) -> np.ndarray:
        n = self.frame_no[stream]
        self.frame_no[stream] = n + 1
        if n > 0:
            c, r = self.ctrl[stream], self.rad[stream]
            u = uniform((self.seed << 20) ^ (stream << 12) ^ n, c.size + r.size + c.size // 2)
            ang = u[:c.size // 2] * 2 * math.pi
            mag = u[c.size // 2:c.size] * 2.0
            c[:, 0::2] += (mag * np.cos(ang)).reshape(c.shape[0], 4)
            c[:, 1::2] += (mag * np.sin(ang)).reshape(c.shape[0], 4)
            r += (u[c.size:c.size + r.size] - 0.5)
            np.clip(r, 1.5, 6.5, out=r)
        return render_strokes2d(self.size, self.size, self.ctrl[stream], self.rad[stream])


def serving_volume(seed: int) -> np.ndarray:
    """Tree volume with sides U[128,320] (tree/ellipsoid counts scaled to volume)."""
    u = uniform(seed, 3)
    s = [int(128 + (320 - 128) * v) for v in u]
    vol = s[0] * s[1] * s[2] / 256 ** 3
    return trees3d(seed, s[0], s[1], s[2], ntrees=max(1, int(round(8 * vol))), nell=int(round(3 * vol)))
