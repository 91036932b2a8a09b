"""Shared test inputs: seeded shapes with an empty outer frame."""
import numpy as np


def clear_frame(a: np.ndarray) -> np.ndarray:
    a = a.copy()
    if a.ndim == 2:
        a[0, :] = a[-1, :] = 0
        a[:, 0] = a[:, -1] = 0
    else:
        a[0] = a[-1] = 0
        a[:, 0] = a[:, -1] = 0
        a[:, :, 0] = a[:, :, -1] = 0
    return a


def random2d(rng, h, w, p):
    return clear_frame((rng.random((h, w)) < p).astype(np.uint8))


def blobs2d(rng, h, w, n, rmax=9):
    yy, xx = np.mgrid[0:h, 0:w]
    a = np.zeros((h, w), np.uint8)
    for _ in range(n):
        cy, cx, r = rng.integers(0, h), rng.integers(0, w), rng.integers(2, rmax)
        a[(yy - cy) ** 2 + (xx - cx) ** 2 <= r * r] = 1
    return clear_frame(a)


def random3d(rng, d, h, w, p):
    return clear_frame((rng.random((d, h, w)) < p).astype(np.uint8))


def blobs3d(rng, d, h, w, n, rmax=6):
    zz, yy, xx = np.mgrid[0:d, 0:h, 0:w]
    a = np.zeros((d, h, w), np.uint8)
    for _ in range(n):
        c = [rng.integers(0, s) for s in (d, h, w)]
        r = rng.integers(2, rmax)
        a[(zz - c[0]) ** 2 + (yy - c[1]) ** 2 + (xx - c[2]) ** 2 <= r * r] = 1
    return clear_frame(a)


def canonical(segs):
    """Canonical form of a segment list: each segment direction-normalised
    (reversed when its last point is smaller than its first), then sorted."""
    out = []
    for is_end, pts in segs:
        p = tuple(pts)
        if p[-1] < p[0]:
            p = tuple(reversed(p))
        out.append((p, is_end))
    return sorted(out)
