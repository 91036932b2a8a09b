"""Serving: every result is the same whether the request ran alone or in the
mix (requests of both lanes in flight together); the tolerance is zero
(thinning is integer work) and each result also equals the oracle."""
import numpy as np
import pytest

from oracle import pyoracle as po
from tests.helpers import blobs2d, blobs3d

pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch
    t = torch.empty(a.shape, dtype=torch.uint8, pin_memory=True)
    t.numpy()[...] = a
    return t


def test_alone_equals_mix():
    import torch
    from begputhinning_b200.serve import Server
    rng = np.random.default_rng(17)
    reqs = []
    for k in range(10):
        if k % 3 == 2:
            reqs.append(blobs3d(rng, *rng.integers(24, 70, 3), 5))
        else:
            reqs.append(blobs2d(rng, *rng.integers(100, 700, 2), 30))
    srv = Server(0, 8 << 30)
    ins = [_pinned(r) for r in reqs]
    alone = []
    for t in ins:
        o = torch.zeros(t.shape, dtype=torch.uint8, pin_memory=True)
        srv.submit(t, o)
        srv.drain(60)
        alone.append(o.numpy().copy())
        srv.poll()
    mixed = [torch.full(t.shape, 9, dtype=torch.uint8, pin_memory=True) for t in ins]
    for t, o in zip(ins, mixed):  # all at once: admitted into slots as they free up
        srv.submit(t, o)
    srv.drain(60)
    done = srv.poll()
    assert len(done) == len(reqs) and all(st == 0 for _, _, st in done)
    for k, (r, a, m) in enumerate(zip(reqs, alone, mixed)):
        assert np.array_equal(a, m.numpy()), f"request {k}: alone and mixed results differ"
        want = po.thin2d(r)[0] if r.ndim == 2 else po.thin3d(r)[0]
        assert np.array_equal(a, want), f"request {k} differs from the oracle"
    s0, s1 = srv.stats(0), srv.stats(1)
    assert s0["completed"] >= 1 and s1["completed"] >= 1
    srv.close()


def test_server_rejects_oversized():
    import torch
    from begputhinning_b200 import BGTError
    from begputhinning_b200.serve import Server
    srv = Server(0, 128 << 20)
    big = torch.zeros((8192, 8192), dtype=torch.uint8)  # 128 MB of staging alone: more than the arena
    with pytest.raises(BGTError):
        srv.submit(big, torch.zeros_like(big))
    srv.close()


def test_admission_waits_for_memory():
    """An arena with room for one volume launch: the other volumes wait
    (not admitted) while it holds the memory and are admitted as it frees;
    frames borrow the room the volumes leave; every output is the oracle's."""
    import time

    import torch
    from begputhinning_b200.serve import Server
    rng = np.random.default_rng(23)
    vols = [blobs3d(rng, 150, 150, 150, 20) for _ in range(3)]
    frames = [blobs2d(rng, 400, 500, 40) for _ in range(4)]
    srv = Server(0, 20 << 20)
    ins = [_pinned(v) for v in vols + frames]
    outs = [torch.full(t.shape, 9, dtype=torch.uint8, pin_memory=True) for t in ins]
    for t, o in zip(ins, outs):
        srv.submit(t, o)
    saw_wait = False
    peak = 0
    done = []
    t_end = time.time() + 60
    while len(done) < len(ins) and time.time() < t_end:
        used, budget, waiting = srv.memory()
        peak = max(peak, used)
        saw_wait |= waiting > 0 and used > 0
        done += srv.poll()
    assert len(done) == len(ins) and all(st == 0 for _, _, st in done)
    assert saw_wait, "no request ever waited for memory"
    assert peak <= budget
    for k, (r, o) in enumerate(zip(vols + frames, outs)):
        want = po.thin2d(r)[0] if r.ndim == 2 else po.thin3d(r)[0]
        assert np.array_equal(o.numpy(), want), f"request {k} differs from the oracle"
    assert srv.memory()[0] == 0
    srv.close()
