"""Python host interface mirroring the reference's C++ entry points.

=========================  ===============================================
reference (C++)            here
=========================  ===============================================
Thinning2D<T>              ``Thinning2D(data) -> out``         (host arrays)
Thinning3D<T>              ``Thinning3D(data) -> out``
CenterlineExtraction<T> 2D ``CenterlineExtraction(data, max_segment_length,
                           smoothing_span) -> (x, y, idx)``
CenterlineExtraction<T> 3D same with a 3-D array -> (x, y, z, idx)
ExtractSegmentsV<T>        ``ExtractSegmentsV(data) -> Segments``
=========================  ===============================================

Argument meaning follows the reference (2D/LibThinning2D.h:14-15,
3D/LibThinning3D.h:14-15, 2D/CenterlineExtraction.h:25-28,
3D/CenterlineExctraction.h:26-29, 2D/ExtractSegments.h:16-17): arrays are
row-major with x fastest, shape (height, width) or (depth, height, width).
Everything runs through libbgt.so; failures raise ``BGTError`` (the
reference had no error channel).  Device-resident variants take torch CUDA
tensors.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import BGTError, check, lib

DTYPES = {
    np.dtype(np.uint8): 0, np.dtype(np.int8): 1, np.dtype(np.uint16): 3, np.dtype(np.int16): 4,
    np.dtype(np.uint32): 5, np.dtype(np.int32): 6, np.dtype(np.float32): 7, np.dtype(np.float64): 8,
    np.dtype(np.bool_): 9,
}


def dtype_code(dt) -> int:
    dt = np.dtype(dt)
    if dt not in DTYPES:
        raise TypeError(f"unsupported pixel type {dt}")
    return DTYPES[dt]


def torch_dtype_code(t) -> int:
    import torch
    m = {torch.uint8: 0, torch.int8: 1, torch.int16: 4, torch.int32: 6, torch.float32: 7,
         torch.float64: 8, torch.bool: 9}
    if hasattr(torch, "uint16"):
        m[torch.uint16] = 3
    if hasattr(torch, "uint32"):
        m[torch.uint32] = 5
    if t.dtype not in m:
        raise TypeError(f"unsupported tensor dtype {t.dtype}")
    return m[t.dtype]


class Context:
    """A device, a stream and resident scratch (bgt_ctx)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().bgt_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            lib().bgt_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream) -> None:
        """Use a torch.cuda.Stream (or raw handle int) for subsequent calls; None = own stream."""
        ptr = None if stream is None else (stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        check(lib().bgt_ctx_set_stream(self.h, ptr))


_default = {}


def default_context(device: int = 0) -> Context:
    if device not in _default:
        _default[device] = Context(device)
    return _default[device]


def _vp(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def Thinning2D(data: np.ndarray, ctx: Context | None = None) -> np.ndarray:
    """Thin a 2-D image (host array). Returns 0/1 in the input's dtype."""
    a = np.ascontiguousarray(data)
    if a.ndim != 2:
        raise ValueError("Thinning2D expects a (height, width) array")
    out = np.empty_like(a)
    ctx = ctx or default_context()
    check(lib().bgt_thin2d(ctx.h, dtype_code(a.dtype), _vp(a), a.shape[1], a.shape[0], _vp(out)))
    return out


def Thinning3D(data: np.ndarray, ctx: Context | None = None) -> np.ndarray:
    """Thin a 3-D volume (host array, shape (depth, height, width))."""
    a = np.ascontiguousarray(data)
    if a.ndim != 3:
        raise ValueError("Thinning3D expects a (depth, height, width) array")
    out = np.empty_like(a)
    ctx = ctx or default_context()
    check(lib().bgt_thin3d(ctx.h, dtype_code(a.dtype), _vp(a), a.shape[2], a.shape[1], a.shape[0], _vp(out)))
    return out


def thin_device(t, out=None, ctx: Context | None = None):
    """Thin a torch CUDA tensor (2-D or 3-D) in stream order; returns `out`."""
    import torch
    t = t.contiguous()
    if out is None:
        out = torch.empty_like(t)
    ctx = ctx or default_context(t.device.index or 0)
    code = torch_dtype_code(t)
    torch.cuda.current_stream().synchronize()
    if t.dim() == 2:
        check(lib().bgt_thin2d_device(ctx.h, code, t.data_ptr(), t.shape[1], t.shape[0], out.data_ptr()))
    elif t.dim() == 3:
        check(lib().bgt_thin3d_device(ctx.h, code, t.data_ptr(), t.shape[2], t.shape[1], t.shape[0],
                                      out.data_ptr()))
    else:
        raise ValueError("expected a 2-D or 3-D tensor")
    torch.cuda.synchronize()
    return out


def _take(ptr, n, dtype):
    if n == 0 or not ptr:
        arr = np.zeros(0, dtype=dtype)
    else:
        arr = np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)
    lib().bgt_free(C.cast(ptr, C.c_void_p))
    return arr


def CenterlineExtraction(data: np.ndarray, max_segment_length: int, smoothing_span: int,
                         ctx: Context | None = None):
    """2-D: returns (x, y, idx); 3-D: (x, y, z, idx).  idx has nsegs+1 entries."""
    a = np.ascontiguousarray(data)
    ctx = ctx or default_context()
    fx, fy, fz = C.POINTER(C.c_float)(), C.POINTER(C.c_float)(), C.POINTER(C.c_float)()
    oi = C.POINTER(C.c_uint)()
    n = C.c_uint()
    if a.ndim == 2:
        check(lib().bgt_centerline2d(ctx.h, dtype_code(a.dtype), _vp(a), a.shape[1], a.shape[0],
                                     int(max_segment_length), int(smoothing_span), C.byref(fx), C.byref(fy),
                                     C.byref(oi), C.byref(n)))
    elif a.ndim == 3:
        check(lib().bgt_centerline3d(ctx.h, dtype_code(a.dtype), _vp(a), a.shape[2], a.shape[1], a.shape[0],
                                     int(max_segment_length), int(smoothing_span), C.byref(fx), C.byref(fy),
                                     C.byref(fz), C.byref(oi), C.byref(n)))
    else:
        raise ValueError("expected a 2-D or 3-D array")
    idx = _take(oi, n.value + 1, np.uint32)
    npts = int(idx[-1])
    x, y = _take(fx, npts, np.float32), _take(fy, npts, np.float32)
    if a.ndim == 3:
        return x, y, _take(fz, npts, np.float32), idx
    return x, y, idx


def matlab_segments(x: np.ndarray, y: np.ndarray, idx: np.ndarray, z: np.ndarray | None = None) -> list:
    """Centreline output in the MATLAB gateways' cell layout: one
    (ssize, 2) array per segment with columns y, x — (ssize, 3) with y, x, z
    in 3-D — in column-major (Fortran) order, doubles; formatted by
    bgt_matlab_segments."""
    dims = 2 if z is None else 3
    idx = np.ascontiguousarray(idx, np.uint32)
    nsegs = len(idx) - 1
    npts = int(idx[-1]) if nsegs >= 0 else 0
    xs = np.ascontiguousarray(x, np.float32)
    ys = np.ascontiguousarray(y, np.float32)
    zs = None if z is None else np.ascontiguousarray(z, np.float32)
    out = np.empty(max(1, dims * npts), np.float64)
    check(lib().bgt_matlab_segments(dims, nsegs, _vp(xs), _vp(ys), None if zs is None else _vp(zs), _vp(idx),
                                    _vp(out)))
    cells = []
    for i in range(nsegs):
        b, n = dims * int(idx[i]), int(idx[i + 1] - idx[i])
        cells.append(out[b:b + dims * n].reshape(n, dims, order="F"))
    return cells


@dataclass
class Segments:
    """ExtractSegmentsV output in emission order."""

    start: np.ndarray   # int32 [nseg+1]
    is_end: np.ndarray  # uint8 [nseg]
    pts: np.ndarray     # int16 [npts, 2 or 3] columns x, y[, z]

    @property
    def nseg(self) -> int:
        return len(self.is_end)

    def as_lists(self):
        out = []
        for k in range(self.nseg):
            p = self.pts[self.start[k]:self.start[k + 1]]
            out.append((int(self.is_end[k]), tuple(map(tuple, p.tolist()))))
        return out


def ExtractSegmentsV(data, ctx: Context | None = None) -> Segments:
    """Segment extraction on the GPU of a thinned image/volume (numpy array or
    torch CUDA tensor); nonzero = foreground as in the reference."""
    import torch
    t = data if isinstance(data, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(data))
    t = t.cuda().contiguous() if not t.is_cuda else t.contiguous()
    ctx = ctx or default_context(t.device.index or 0)
    code = torch_dtype_code(t)
    st = C.POINTER(C.c_int32)()
    ie = C.POINTER(C.c_uint8)()
    px, py, pz = C.POINTER(C.c_int16)(), C.POINTER(C.c_int16)(), C.POINTER(C.c_int16)()
    ns, npt = C.c_int(), C.c_int()
    torch.cuda.current_stream(t.device).synchronize()
    if t.dim() == 2:
        check(lib().bgt_segments2d_device(ctx.h, code, t.data_ptr(), t.shape[1], t.shape[0], C.byref(st),
                                          C.byref(ie), C.byref(px), C.byref(py), C.byref(ns), C.byref(npt)))
        dims = 2
    else:
        check(lib().bgt_segments3d_device(ctx.h, code, t.data_ptr(), t.shape[2], t.shape[1], t.shape[0],
                                          C.byref(st), C.byref(ie), C.byref(px), C.byref(py), C.byref(pz),
                                          C.byref(ns), C.byref(npt)))
        dims = 3
    n, m = ns.value, npt.value
    start = _take(st, n + 1, np.int32)
    is_end = _take(ie, n, np.uint8)
    cols = [_take(px, m, np.int16), _take(py, m, np.int16)]
    if dims == 3:
        cols.append(_take(pz, m, np.int16))
    pts = np.stack(cols, axis=1) if m else np.zeros((0, dims), np.int16)
    return Segments(start, is_end, pts)


class Batch:
    """Many images/volumes thinned together by the persistent engine.

    >>> b = Batch(ctx); ids = [b.add(t.shape) for t in tensors]; b.finalize()
    >>> for i, t in zip(ids, tensors): b.set_io(i, t, out[i])
    >>> b.run()            # persistent engine (mode 0); b.run(plain=True) for the plain path
    """

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        check(lib().bgt_batch_create(self.ctx.h, C.byref(h)))
        self.h = h
        self.shapes = []
        self._keep = {}

    def add(self, shape, cfg: int = -1) -> int:
        i = C.c_int()
        if len(shape) == 2:
            check(lib().bgt_batch_add2d(self.h, shape[1], shape[0], cfg, C.byref(i)))
        else:
            check(lib().bgt_batch_add3d(self.h, shape[2], shape[1], shape[0], cfg, C.byref(i)))
        self.shapes.append(tuple(shape))
        return i.value

    def set_grid(self, ctas: int) -> None:
        """Cap the persistent engine's grid at `ctas` CTAs (0: no cap);
        call before finalize()."""
        check(lib().bgt_batch_set_grid(self.h, ctas))

    def set_engine(self, rings_only: bool) -> None:
        """Thin every instance with the tile rings (True) or let the
        resident kernel take every instance that fits (False, the default);
        call before finalize()."""
        check(lib().bgt_batch_set_engine(self.h, 1 if rings_only else 0))

    def plan(self, i: int):
        """(resident, bands): whether the resident kernel takes instance i
        and how many CTAs a 2D image is cut into."""
        r, n = C.c_int(), C.c_int()
        check(lib().bgt_batch_plan(self.h, i, C.byref(r), C.byref(n)))
        return bool(r.value), n.value

    def finalize(self) -> None:
        check(lib().bgt_batch_finalize(self.h))

    def set_io(self, i: int, t_in, t_out=None) -> None:
        """Device input tensor and (optional) output tensor of the same shape/dtype."""
        self._keep[i] = (t_in, t_out)
        check(lib().bgt_batch_set_io(self.h, i, torch_dtype_code(t_in), t_in.data_ptr(),
                                     t_out.data_ptr() if t_out is not None else None))

    def run(self, plain: bool = False, graph: bool = True, sync: bool = True, device_loop: bool = False) -> None:
        """Run the batch on the context's stream.  With sync (default) the
        caller's torch stream is drained first and the device is synchronised
        after, so torch tensors can be used directly before and after.
        `plain` runs one launch per pass per instance; with `device_loop` the
        pass loop of the plain path stays on the device (a CUDA graph with a
        conditional node per instance) instead of reading the change flag
        back after every pass."""
        if sync:
            import torch
            torch.cuda.current_stream().synchronize()
        mode = (2 if device_loop else 1) if plain else 0
        check(lib().bgt_batch_run(self.h, mode, 0 if plain else int(graph)))
        if sync:
            import torch
            torch.cuda.synchronize()

    def stats(self, i: int):
        p, c, g = C.c_int(), C.c_int(), C.c_int()
        check(lib().bgt_batch_instance_stats(self.h, i, C.byref(p), C.byref(c), C.byref(g)))
        return {"passes": p.value, "converged": c.value, "cfg": g.value}

    def work(self):
        """(tiles processed, packed core words processed) of the last run."""
        t, w = C.c_ulonglong(), C.c_ulonglong()
        check(lib().bgt_batch_work(self.h, C.byref(t), C.byref(w)))
        return t.value, w.value

    def stage_ms(self):
        """(pack, engine, unpack) device milliseconds of the last engine run."""
        a, b, c = C.c_float(), C.c_float(), C.c_float()
        check(lib().bgt_batch_stage_ms(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def res_trace(self):
        """Per work item of the resident kernel's last run, in the order taken:
        (instance, band, start ns, end ns, SM)."""
        n = C.c_int()
        check(lib().bgt_batch_res_trace(self.h, C.byref(n), None, None, None, None, None, 0))
        m = n.value
        if m == 0:
            return []
        inst, band, sm = (C.c_int * m)(), (C.c_int * m)(), (C.c_int * m)()
        t0, t1 = (C.c_longlong * m)(), (C.c_longlong * m)()
        check(lib().bgt_batch_res_trace(self.h, C.byref(n), inst, band, t0, t1, sm, m))
        return list(zip(inst, band, t0, t1, sm))

    def engine_ms(self):
        """(resident kernel, tile rings) device milliseconds of the last engine run."""
        a, b = C.c_float(), C.c_float()
        check(lib().bgt_batch_engine_ms(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def device_bytes(self) -> int:
        n = C.c_size_t()
        check(lib().bgt_batch_device_bytes(self.h, C.byref(n)))
        return n.value

    def close(self):
        if self.h:
            lib().bgt_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PipelinedBatch:
    """Host-to-host thinning of many instances with transfers overlapped.

    The instances (in the given order, as contiguous byte ranges of one
    uint8 host input and one host output, both pinned) are split into
    `chunks` consecutive groups of similar size.  Each group is a Batch of
    its own; group c is copied in on a copy stream, thinned on the compute
    stream once its copy finished, and copied out on a third stream, so the
    copy-in of later groups and the copy-out of earlier ones run during the
    thinning of the current group.  Put instances with long chains of passes
    (3D volumes) first: their group starts first.

    `buffers` device copies of the inputs and outputs are used in turn by
    consecutive passes, so the copy-in of pass k+1 runs while pass k is still
    being thinned and copied out (host-to-device and device-to-host copies
    use the two directions of the link at the same time).  A device buffer is
    overwritten only after the copy-out of the pass that last used it."""

    def __init__(self, shapes, chunks: int = 4, device: int = 0, buffers: int = 2):
        import numpy as np
        import torch
        if buffers < 1:
            raise ValueError("buffers must be >= 1")
        self.device = device
        self.dev = torch.device("cuda", device)
        self.shapes = [tuple(s) for s in shapes]
        sizes = [int(np.prod(s)) for s in self.shapes]
        self.offs = np.cumsum([0] + sizes)
        self.total = int(self.offs[-1])
        target = self.total / max(1, chunks)
        bounds, acc, start = [], 0, 0
        for i, s in enumerate(sizes):
            acc += s
            if acc >= target * (len(bounds) + 1) and len(bounds) < chunks - 1:
                bounds.append((start, i + 1))
                start = i + 1
        if start < len(sizes):
            bounds.append((start, len(sizes)))
        self.groups = bounds
        self.s_in = torch.cuda.Stream(self.dev)
        self.s_comp = torch.cuda.Stream(self.dev)
        self.s_out = torch.cuda.Stream(self.dev)
        self.ctx = Context(device)
        self.ctx.set_stream(self.s_comp)
        self.sets = []  # per device buffer: (dev_in, dev_out, batches)
        for _ in range(buffers):
            dev_in = torch.empty(self.total, dtype=torch.uint8, device=self.dev)
            dev_out = torch.empty(self.total, dtype=torch.uint8, device=self.dev)
            batches = []
            for a, b in self.groups:
                bt = Batch(self.ctx)
                ids = [bt.add(self.shapes[i]) for i in range(a, b)]
                bt.finalize()
                for j, i in zip(ids, range(a, b)):
                    lo, hi = int(self.offs[i]), int(self.offs[i + 1])
                    bt.set_io(j, dev_in[lo:hi], dev_out[lo:hi])
                batches.append(bt)
            self.sets.append((dev_in, dev_out, batches))
        self.free = [None] * buffers  # event: the set's last copy-out finished
        self.turn = 0
        torch.cuda.synchronize(self.dev)

    @property
    def dev_in(self):
        return self.sets[0][0]

    @property
    def dev_out(self):
        return self.sets[0][1]

    @property
    def batches(self):
        return self.sets[0][2]

    def run(self, host_in, host_out) -> None:
        """Enqueue one host-to-host pass (no synchronisation).  The caller
        keeps `host_in` unchanged and does not read `host_out` until the
        pass's copies finished (e.g. `torch.cuda.synchronize()`)."""
        import torch
        k = self.turn % len(self.sets)
        self.turn += 1
        dev_in, dev_out, batches = self.sets[k]
        if self.free[k] is not None:
            self.s_in.wait_event(self.free[k])
        for (a, b), bt in zip(self.groups, batches):
            lo, hi = int(self.offs[a]), int(self.offs[b])
            e_in = torch.cuda.Event()
            with torch.cuda.stream(self.s_in):
                dev_in[lo:hi].copy_(host_in[lo:hi], non_blocking=True)
                e_in.record(self.s_in)
            self.s_comp.wait_event(e_in)
            bt.run(graph=True, sync=False)
            e_c = torch.cuda.Event()
            e_c.record(self.s_comp)
            self.s_out.wait_event(e_c)
            with torch.cuda.stream(self.s_out):
                host_out[lo:hi].copy_(dev_out[lo:hi], non_blocking=True)
        e_end = torch.cuda.Event()
        e_end.record(self.s_out)
        self.free[k] = e_end

    def close(self):
        for _, _, batches in self.sets:
            for bt in batches:
                bt.close()
        self.sets = []
        self.ctx.close()


def cfg_list(dims: int):
    ids = (C.c_int * 32)()
    n = C.c_int()
    check(lib().bgt_cfg_list(dims, ids, 32, C.byref(n)))
    return [ids[i] for i in range(n.value)]


def cfg_describe(cfg: int) -> dict:
    v = [C.c_int() for _ in range(6)]
    check(lib().bgt_cfg_describe(cfg, *[C.byref(x) for x in v]))
    return dict(zip(["dims", "k", "tw", "th", "tz", "smem"], [x.value for x in v]))


__all__ = ["BGTError", "Context", "default_context", "Thinning2D", "Thinning3D", "thin_device",
           "CenterlineExtraction", "ExtractSegmentsV", "Segments", "Batch", "cfg_list", "cfg_describe",
           "dtype_code", "torch_dtype_code"]
