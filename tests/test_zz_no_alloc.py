"""The no-allocation thinning entry point (bgt_thin2d_device_noalloc).

It serves callers that cannot allocate device memory (a plugin inside an
application that owns all device memory through its own pool, a real-time
loop that cannot afford an allocation's implicit synchronisation), so it
runs on a scratch array compiled into the library.  This test calls it
through the C ABI twice in a row, on different images, and checks each
output bit for bit (thinning is integer work, the tolerance is zero)
against the allocating entry point bgt_thin2d_device and against the
oracle.  The file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as po
from tests.helpers import blobs2d

pytestmark = pytest.mark.gpu


def _reference_thin(ctx, t):
    import torch
    from begputhinning_b200 import lib
    out = torch.zeros_like(t)
    torch.cuda.synchronize()
    rc = lib().bgt_thin2d_device(ctx.h, 0, t.data_ptr(), t.shape[1], t.shape[0], out.data_ptr())
    assert rc == 0, lib().bgt_last_error()
    torch.cuda.synchronize()
    return out


def test_noalloc_matches_allocating_path():
    import torch
    from begputhinning_b200 import Context, lib
    ctx = Context(0)
    rng = np.random.default_rng(99)
    images = [blobs2d(rng, 300, 410, 40), blobs2d(rng, 1031, 777, 120)]
    stream = torch.cuda.Stream()
    for img in images:  # two calls in a row; the second reuses the array the first left behind
        t = torch.from_numpy(img).cuda()
        out = torch.full_like(t, 7)
        torch.cuda.synchronize()
        rc = lib().bgt_thin2d_device_noalloc(0, 0, C.c_void_p(t.data_ptr()), img.shape[1], img.shape[0],
                                             C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == 0, lib().bgt_last_error()
        want = _reference_thin(ctx, t)
        assert torch.equal(out, want), f"shape {img.shape}: {(out != want).sum().item()} pixels differ"
        assert np.array_equal(out.cpu().numpy(), po.thin2d(img)[0]), f"shape {img.shape}: differs from the oracle"
    ctx.close()


def test_noalloc_rejects_oversized_images():
    import torch
    from begputhinning_b200 import lib
    big = torch.zeros((8192, 8192), dtype=torch.uint8, device="cuda")
    rc = lib().bgt_thin2d_device_noalloc(0, 0, C.c_void_p(big.data_ptr()), 8192, 8192,
                                         C.c_void_p(big.data_ptr()), None)
    assert rc == 5  # BGT_ERR_LIMIT
    assert b"scratch" in lib().bgt_last_error()
