"""MATLAB column-order formatting of centreline output (bgt_matlab_segments)
against the cell layout the reference's MEX gateways build
(2D/Matlab2DThinning.cpp:163-175, 3D/Matlab3DThinning.cpp:157-171): per
segment an ssize x dims double matrix, column-major, columns y, x (, z)."""
import numpy as np
import pytest

from begputhinning_b200 import matlab_segments


def gateway_cells(x, y, idx, z=None):
    """The gateway's loop, restated: ds[ti] = y, ds[ssize + ti] = x, ds[2*ssize + ti] = z."""
    cols = 2 if z is None else 3
    cells = []
    for i in range(len(idx) - 1):
        ssize = int(idx[i + 1] - idx[i])
        ds = np.zeros(ssize * cols, np.float64)
        for ti, pi in enumerate(range(int(idx[i]), int(idx[i + 1]))):
            ds[ti] = float(y[pi])
            ds[ssize + ti] = float(x[pi])
            if z is not None:
                ds[2 * ssize + ti] = float(z[pi])
        cells.append(ds.reshape(ssize, cols, order="F"))
    return cells


@pytest.mark.parametrize("dims", [2, 3])
def test_matlab_segments_match_gateway_layout(dims):
    rng = np.random.default_rng(7)
    lens = rng.integers(1, 40, size=25)
    idx = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)
    n = int(idx[-1])
    x = (rng.random(n) * 500).astype(np.float32)
    y = (rng.random(n) * 500).astype(np.float32)
    z = (rng.random(n) * 500).astype(np.float32) if dims == 3 else None
    got = matlab_segments(x, y, idx, z)
    want = gateway_cells(x, y, idx, z)
    assert len(got) == len(want) == 25
    for g, w in zip(got, want):
        assert g.shape == w.shape
        assert np.array_equal(g, w)


def test_matlab_segments_empty():
    assert matlab_segments(np.zeros(0, np.float32), np.zeros(0, np.float32), np.zeros(1, np.uint32)) == []
