"""CPU: the seeded generators are deterministic, clear the outer frame and
produce the workload shapes."""
import numpy as np

from begputhinning_b200 import synth


def _frame_clear(a):
    if a.ndim == 2:
        return not (a[0].any() or a[-1].any() or a[:, 0].any() or a[:, -1].any())
    return not (a[0].any() or a[-1].any() or a[:, 0].any() or a[:, -1].any() or a[:, :, 0].any()
                or a[:, :, -1].any())


def test_deterministic_and_frame():
    a = synth.frame512(0)
    b = synth.frame512(0)
    assert np.array_equal(a, b) and a.shape == (512, 512) and a.dtype == np.uint8
    assert _frame_clear(a) and 0.02 < a.mean() < 0.4
    assert not np.array_equal(a, synth.frame512(1))
    v = synth.trees3d(3, 64, 48, 40, ntrees=2, nell=1)
    assert v.shape == (40, 48, 64) and _frame_clear(v) and v.any()
    ves = synth.vessels2d(1, 512, 384, nroots=4)
    assert _frame_clear(ves) and 0.005 < ves.mean() < 0.3


def test_mixed_batch_shapes():
    s2, s3 = synth.mixed_batch_shapes(3)
    assert len(s2) == 512 and len(s3) == 32
    assert all(64 <= w <= 2048 and 64 <= h <= 2048 and n >= 1 for w, h, n in s2)
    assert all(64 <= a <= 192 and 64 <= b <= 192 and 64 <= c <= 192 for a, b, c, _, _ in s3)
    px = sum(w * h for w, h, _ in s2)
    assert 2.0e8 < px < 5.0e8


def test_frame_streams_correlated():
    fs = synth.FrameStreams(seed=4, streams=2, size=256, strokes=6)
    f0 = fs.next(0)
    f1 = fs.next(0)
    assert f0.shape == (256, 256) and _frame_clear(f1)
    # consecutive frames of a stream overlap strongly (strokes move <= 2 px)
    inter = np.logical_and(f0, f1).sum() / max(1, np.logical_or(f0, f1).sum())
    assert inter > 0.4
