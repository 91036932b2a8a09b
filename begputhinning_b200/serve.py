"""Serving: the native request loop (bgt_server_* in libbgt.so) and a
Poisson load generator for the mixed frame/volume workload.

Workload: 16 concurrent streams of 1024x1024 frames at 30 fps (strokes
displaced <= 2 px per frame, radius jitter +/-0.5 px) are 70% of the
requests; tree volumes with sides U[128,320] are the other 30%.  Arrivals
are a Poisson process at the combined rate (480 frames/s / 0.7).  Device
memory is one resident arena of the HBM budget (64 GB by default); the
runtime admits a request when a slot of its lane is free and the arena has
room for it, and frees the memory when its output is back in host memory.
Latency is measured per request from submission to output in host memory."""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from ._lib import check, lib
from .api import dtype_code
from . import synth


class Server:
    def __init__(self, device: int = 0, hbm_budget_bytes: int = 64 << 30):
        h = C.c_void_p()
        check(lib().bgt_server_create(device, hbm_budget_bytes, C.byref(h)))
        self.h = h
        self._keep = {}

    def submit(self, host_in, host_out) -> int:
        """host_in/host_out: pinned torch CPU tensors or numpy arrays of shape
        (H, W) or (D, H, W); both must stay alive until completion."""
        a = host_in.numpy() if hasattr(host_in, "numpy") else host_in
        shape = a.shape
        w, h, d = (shape[1], shape[0], 1) if len(shape) == 2 else (shape[2], shape[1], shape[0])
        t = C.c_ulonglong()
        check(lib().bgt_server_submit(self.h, dtype_code(a.dtype), C.c_void_p(_ptr(host_in)), w, h, d,
                                      C.c_void_p(_ptr(host_out)), C.byref(t)))
        self._keep[t.value] = (host_in, host_out)
        return t.value

    def poll(self, cap: int = 4096):
        tk = (C.c_ulonglong * cap)()
        lat = (C.c_double * cap)()
        st = (C.c_int * cap)()
        n = C.c_int()
        check(lib().bgt_server_poll(self.h, tk, lat, st, cap, C.byref(n)))
        out = []
        for i in range(n.value):
            self._keep.pop(tk[i], None)
            out.append((tk[i], lat[i], st[i]))
        return out

    def drain(self, timeout_s: float = 60.0) -> None:
        check(lib().bgt_server_drain(self.h, timeout_s))

    def stats(self, lane: int) -> dict:
        p50, p99, thr = C.c_double(), C.c_double(), C.c_double()
        n = C.c_ulonglong()
        check(lib().bgt_server_stats(self.h, lane, C.byref(p50), C.byref(p99), C.byref(thr), C.byref(n)))
        return {"p50_ms": p50.value, "p99_ms": p99.value, "mvoxel_per_s": thr.value, "completed": n.value}

    def reset_stats(self) -> None:
        check(lib().bgt_server_reset_stats(self.h))

    def memory(self):
        """(arena bytes held by launches in flight, arena bytes, requests waiting for admission)"""
        u, b, w = C.c_size_t(), C.c_size_t(), C.c_ulonglong()
        check(lib().bgt_server_memory(self.h, C.byref(u), C.byref(b), C.byref(w)))
        return u.value, b.value, w.value

    def close(self):
        if self.h:
            lib().bgt_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr(x) -> int:
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    return x.ctypes.data


def _pinned(arr: np.ndarray):
    import torch
    t = torch.empty(arr.shape, dtype=torch.uint8, pin_memory=True)
    t.numpy()[...] = arr
    return t


def run_workload(duration_s: float = 3.0, seed: int = 4, streams: int = 16, fps: float = 30.0,
                 frame_share: float = 0.7, volumes: int = 12, device: int = 0, budget: int = 64 << 30,
                 warmup_s: float = 0.5) -> dict:
    """Drive a Server with Poisson arrivals; returns latency and throughput per lane."""
    import torch
    gen = synth.FrameStreams(seed=seed, streams=streams, size=1024)
    per_stream = 8
    frames = [[_pinned(gen.next(s)) for _ in range(per_stream)] for s in range(streams)]
    vols = [_pinned(synth.serving_volume(seed * 7919 + k)) for k in range(volumes)]
    frame_rate = streams * fps
    rate = frame_rate / frame_share
    u = synth.uniform(seed + 12345, 3 * int(rate * (duration_s + warmup_s) * 1.5 + 100))
    srv = Server(device, budget)
    outs_f = [torch.empty((1024, 1024), dtype=torch.uint8, pin_memory=True) for _ in range(96)]
    outs_v = {k: [torch.empty(v.shape, dtype=torch.uint8, pin_memory=True) for _ in range(6)]
              for k, v in enumerate(vols)}
    free_f = list(range(len(outs_f)))
    free_v = {k: list(range(6)) for k in outs_v}
    owner = {}
    t0 = time.perf_counter()
    t = 0.0
    k = 0
    frame_no = [0] * streams
    sent = {"frames": 0, "volumes": 0}
    stats_reset = False
    total = duration_s + warmup_s
    while True:
        t += -math.log(max(1e-12, u[k])) / rate
        kind = u[k + 1] < frame_share
        pick = u[k + 2]
        k += 3
        if t > total:
            break
        while time.perf_counter() - t0 < t:
            for tk, _, _ in srv.poll():
                typ, idx, slot = owner.pop(tk)
                (free_f if typ == "f" else free_v[idx]).append(slot)
        if not stats_reset and t >= warmup_s:
            srv.reset_stats()
            stats_reset = True
        if kind:
            s = int(pick * streams) % streams
            src = frames[s][frame_no[s] % per_stream]
            frame_no[s] += 1
            while not free_f:
                for tk, _, _ in srv.poll():
                    typ, idx, slot = owner.pop(tk)
                    (free_f if typ == "f" else free_v[idx]).append(slot)
            slot = free_f.pop()
            tk = srv.submit(src, outs_f[slot])
            owner[tk] = ("f", 0, slot)
            sent["frames"] += 1
        else:
            vi = int(pick * len(vols)) % len(vols)
            while not free_v[vi]:
                for tk, _, _ in srv.poll():
                    typ, idx, slot = owner.pop(tk)
                    (free_f if typ == "f" else free_v[idx]).append(slot)
            slot = free_v[vi].pop()
            tk = srv.submit(vols[vi], outs_v[vi][slot])
            owner[tk] = ("v", vi, slot)
            sent["volumes"] += 1
    srv.drain(120.0)
    wall = time.perf_counter() - t0
    res = {"frames": srv.stats(0), "volumes": srv.stats(1), "sent": sent, "wall_s": wall,
           "offered_rate_per_s": rate, "duration_s": duration_s, "warmup_s": warmup_s}
    srv.close()
    return res
