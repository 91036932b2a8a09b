"""ctypes bindings for the oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/liboracle.so`` (the CPU restatement of the reference's hot
path) and, where present, ``oracle/_ref/libref{2d,3d}.so`` (the reference's
own host code and rule functions) and ``oracle/_ref/libref{2d,3d}_gpu.so``
(the reference's CUDA library rebuilt for sm_100a).  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU baseline may import this
module; the product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


class _Segs(C.Structure):
    _fields_ = [
        ("nseg", C.c_int32),
        ("npts", C.c_int32),
        ("start", C.POINTER(C.c_int32)),
        ("is_end", C.POINTER(C.c_uint8)),
        ("x", C.POINTER(C.c_int16)),
        ("y", C.POINTER(C.c_int16)),
        ("z", C.POINTER(C.c_int16)),
    ]


class _CL(C.Structure):
    _fields_ = [
        ("nsegs", C.c_uint32),
        ("npts", C.c_uint32),
        ("x", C.POINTER(C.c_float)),
        ("y", C.POINTER(C.c_float)),
        ("z", C.POINTER(C.c_float)),
        ("idx", C.POINTER(C.c_uint32)),
    ]


@dataclass
class Segments:
    """Segment list in emission order: start offsets, is_end flags, points."""

    start: np.ndarray  # int32 [nseg+1]
    is_end: np.ndarray  # uint8 [nseg]
    pts: np.ndarray  # int16 [npts, 2 or 3] columns x, y[, z]

    @property
    def nseg(self) -> int:
        return len(self.is_end)

    def as_lists(self):
        """[(is_end, tuple(points))] in emission order."""
        out = []
        for k in range(self.nseg):
            p = self.pts[self.start[k]:self.start[k + 1]]
            out.append((int(self.is_end[k]), tuple(map(tuple, p.tolist()))))
        return out


@dataclass
class Centerline:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray | None
    idx: np.ndarray

    @property
    def nsegs(self) -> int:
        return len(self.idx) - 1


def _arr(ptr, n, dtype):
    if n == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def build(ref: bool = False) -> None:
    """Compile liboracle.so (and the _ref libraries when ref=True)."""
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        u8p = C.POINTER(C.c_uint8)
        L.oracle_thin2d.argtypes = [u8p, C.c_int, C.c_int, C.c_int]
        L.oracle_thin3d.argtypes = [u8p, C.c_int, C.c_int, C.c_int, C.c_int]
        L.oracle_segments2d.argtypes = [u8p, C.c_int, C.c_int, C.POINTER(_Segs)]
        L.oracle_segments3d.argtypes = [u8p, C.c_int, C.c_int, C.c_int, C.POINTER(_Segs)]
        L.oracle_segs_free.argtypes = [C.POINTER(_Segs)]
        L.oracle_centerline2d.argtypes = [u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_CL)]
        L.oracle_centerline3d.argtypes = [u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          C.POINTER(_CL)]
        L.oracle_prune_smooth.argtypes = [C.POINTER(_Segs), C.c_int, C.c_int, C.c_int, C.POINTER(_CL)]
        L.oracle_cl_free.argtypes = [C.POINTER(_CL)]
        L.oracle_binarise.argtypes = [C.c_int, C.c_void_p, C.c_int64, C.c_int, u8p]
        L.oracle_rule_table.argtypes = [C.c_int, C.c_int, C.c_void_p]
        L.oracle_rule2d.argtypes = [C.c_int, C.POINTER(C.c_uint64)]
        L.oracle_rule2d.restype = C.c_uint64
        L.oracle_rule3d.argtypes = [C.c_int, C.POINTER(C.c_uint64)]
        L.oracle_rule3d.restype = C.c_uint64
        _lib = L
    return _lib


def _u8(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def thin2d(img: np.ndarray, nthreads: int = 0) -> tuple[np.ndarray, int]:
    """Global synchronous 2D thinning of an (h, w) image. Returns (mask u8, iterations)."""
    a = np.ascontiguousarray(img != 0, dtype=np.uint8)
    h, w = a.shape
    it = lib().oracle_thin2d(_u8(a), w, h, nthreads)
    return a, it


def thin3d(vol: np.ndarray, nthreads: int = 0) -> tuple[np.ndarray, int]:
    """Global synchronous 3D thinning of a (d, h, w) volume. Returns (mask u8, iterations)."""
    a = np.ascontiguousarray(vol != 0, dtype=np.uint8)
    d, h, w = a.shape
    it = lib().oracle_thin3d(_u8(a), w, h, d, nthreads)
    return a, it


def _take_segs(s: _Segs, dims: int, free) -> Segments:
    n, npts = s.nseg, s.npts
    start = _arr(s.start, n + 1, np.int32)
    is_end = _arr(s.is_end, n, np.uint8)
    cols = [_arr(s.x, npts, np.int16), _arr(s.y, npts, np.int16)]
    if dims == 3:
        cols.append(_arr(s.z, npts, np.int16))
    free(C.byref(s))
    pts = np.stack(cols, axis=1) if npts else np.zeros((0, dims), np.int16)
    if n == 0:
        start = np.zeros(1, np.int32)
    return Segments(start, is_end, pts)


def segments2d(img: np.ndarray) -> Segments:
    a = np.ascontiguousarray(img != 0, dtype=np.uint8)
    h, w = a.shape
    s = _Segs()
    lib().oracle_segments2d(_u8(a), w, h, C.byref(s))
    return _take_segs(s, 2, lib().oracle_segs_free)


def segments3d(vol: np.ndarray) -> Segments:
    a = np.ascontiguousarray(vol != 0, dtype=np.uint8)
    d, h, w = a.shape
    s = _Segs()
    lib().oracle_segments3d(_u8(a), w, h, d, C.byref(s))
    return _take_segs(s, 3, lib().oracle_segs_free)


def _take_cl(c: _CL, dims: int, free) -> Centerline:
    n, npts = c.nsegs, c.npts
    out = Centerline(
        _arr(c.x, npts, np.float32),
        _arr(c.y, npts, np.float32),
        _arr(c.z, npts, np.float32) if dims == 3 else None,
        _arr(c.idx, n + 1, np.uint32),
    )
    free(C.byref(c))
    return out


def centerline2d(img: np.ndarray, max_segment_length: int, smoothing_span: int,
                 nthreads: int = 0) -> Centerline:
    a = np.ascontiguousarray(img != 0, dtype=np.uint8)
    h, w = a.shape
    c = _CL()
    lib().oracle_centerline2d(_u8(a), w, h, max_segment_length, smoothing_span, nthreads, C.byref(c))
    return _take_cl(c, 2, lib().oracle_cl_free)


def centerline3d(vol: np.ndarray, max_segment_length: int, smoothing_span: int,
                 nthreads: int = 0) -> Centerline:
    a = np.ascontiguousarray(vol != 0, dtype=np.uint8)
    d, h, w = a.shape
    c = _CL()
    lib().oracle_centerline3d(_u8(a), w, h, d, max_segment_length, smoothing_span, nthreads, C.byref(c))
    return _take_cl(c, 3, lib().oracle_cl_free)


def prune_smooth(segs: Segments, dims: int, max_segment_length: int, smoothing_span: int) -> Centerline:
    """Host tail of CenterlineExtraction applied to an existing segment list."""
    n = segs.nseg
    start = np.ascontiguousarray(segs.start, np.int32)
    is_end = np.ascontiguousarray(segs.is_end, np.uint8)
    cols = [np.ascontiguousarray(segs.pts[:, k], np.int16) for k in range(dims)]
    s = _Segs()
    s.nseg, s.npts = n, int(segs.pts.shape[0])
    s.start = start.ctypes.data_as(C.POINTER(C.c_int32))
    s.is_end = is_end.ctypes.data_as(C.POINTER(C.c_uint8))
    s.x = cols[0].ctypes.data_as(C.POINTER(C.c_int16))
    s.y = cols[1].ctypes.data_as(C.POINTER(C.c_int16))
    s.z = cols[2].ctypes.data_as(C.POINTER(C.c_int16)) if dims == 3 else C.POINTER(C.c_int16)()
    c = _CL()
    lib().oracle_prune_smooth(C.byref(s), dims, max_segment_length, smoothing_span, C.byref(c))
    return _take_cl(c, dims, lib().oracle_cl_free)


def binarise(arr: np.ndarray, dtype_code: int, dims: int) -> np.ndarray:
    a = np.ascontiguousarray(arr)
    out = np.empty(a.shape, np.uint8)
    rc = lib().oracle_binarise(dtype_code, a.ctypes.data_as(C.c_void_p), a.size, dims, _u8(out))
    assert rc == 0
    return out


def rule2d(direction: int, x8: np.ndarray) -> np.ndarray:
    """Deletable mask for N,S,E,W (0..3) given x8 = uint64[8] N,NE,E,SE,S,SW,W,NW."""
    a = np.ascontiguousarray(x8, np.uint64)
    return np.uint64(lib().oracle_rule2d(direction, a.ctypes.data_as(C.POINTER(C.c_uint64))))


def rule3d(direction: int, nb27: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(nb27, np.uint64)
    return np.uint64(lib().oracle_rule3d(direction, a.ctypes.data_as(C.POINTER(C.c_uint64))))


def rule_table(dims: int, direction: int) -> np.ndarray:
    """Deletable-set table of one direction over every neighbourhood
    (uint32[8] in 2D, uint32[2^21] in 3D; layout of bgt_rule_table)."""
    out = np.zeros(8 if dims == 2 else 1 << 21, np.uint32)
    lib().oracle_rule_table(dims, direction, out.ctypes.data_as(C.c_void_p))
    return out


def rule3d_exhaustive_vs_ref(direction: int) -> int:
    """Bits on which the restated 3D rule and the reference's own rule
    function differ, over all 2^26 neighbourhoods (needs oracle/_ref)."""
    L = lib()
    L.oracle_rule3d_exhaustive.argtypes = [C.c_int, C.c_void_p]
    L.oracle_rule3d_exhaustive.restype = C.c_longlong
    fn = C.cast(ref("3d").ref3d_rule, C.c_void_p)
    return int(L.oracle_rule3d_exhaustive(direction, fn))


# --------------------------------------------------------------------------
# The reference's own code (built only where the reference tree exists).
# --------------------------------------------------------------------------
_ref = {}


def have_ref(which: str = "2d") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref{which}.so"))


def ref(which: str):
    if which not in _ref:
        L = C.CDLL(os.path.join(REF_DIR, f"libref{which}.so"))
        u8p = C.POINTER(C.c_uint8)
        if which == "2d":
            L.ref2d_rule.argtypes = [C.c_int, C.c_uint32, C.c_uint32, C.c_uint32]
            L.ref2d_rule.restype = C.c_uint32
            L.ref2d_thin_u8.argtypes = [C.c_int, C.c_int, u8p, u8p]
            L.ref2d_segments_u8.argtypes = [u8p, C.c_int, C.c_int, C.POINTER(_Segs)]
            L.ref2d_centerline.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.POINTER(C.c_float)),
                                           C.POINTER(C.POINTER(C.c_uint32))]
            L.ref2d_centerline.restype = C.c_uint32
        elif which == "3d":
            L.ref3d_rule.argtypes = [C.c_int, C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32]
            L.ref3d_rule.restype = C.c_uint32
            L.ref3d_thin_u8.argtypes = [C.c_int, C.c_int, C.c_int, u8p, u8p]
            L.ref3d_segments_u8.argtypes = [u8p, C.c_int, C.c_int, C.c_int, C.POINTER(_Segs)]
            L.ref3d_centerline.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.POINTER(C.c_float)),
                                           C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.POINTER(C.c_uint32))]
            L.ref3d_centerline.restype = C.c_uint32
        elif which == "2d_gpu":
            L.ref2d_gpu_thin_u8.argtypes = [C.c_int, C.c_int, u8p, u8p]
        elif which == "3d_gpu":
            L.ref3d_gpu_thin_u8.argtypes = [C.c_int, C.c_int, C.c_int, u8p, u8p]
        if which in ("2d", "3d"):
            L.ref_segs_free.argtypes = [C.POINTER(_Segs)]
            L.ref_free_f32.argtypes = [C.POINTER(C.c_float)]
            L.ref_free_u32.argtypes = [C.POINTER(C.c_uint32)]
        _ref[which] = L
    return _ref[which]


def ref_thin2d(img: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(img != 0, dtype=np.uint8)
    h, w = a.shape
    out = np.zeros_like(a)
    ref("2d").ref2d_thin_u8(w, h, _u8(a), _u8(out))
    return out


def ref_thin3d(vol: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(vol != 0, dtype=np.uint8)
    d, h, w = a.shape
    out = np.zeros_like(a)
    ref("3d").ref3d_thin_u8(w, h, d, _u8(a), _u8(out))
    return out


def ref_gpu_thin2d(img: np.ndarray) -> np.ndarray:
    """The reference's own CUDA 2D library (safe only for widths <= 1024)."""
    a = np.ascontiguousarray(img != 0, dtype=np.uint8)
    h, w = a.shape
    if w > 1024:
        raise ValueError("the reference 2D kernel is out of bounds for widths above 1024")
    if h <= 64:
        raise ValueError("the reference 2D launcher sizes an empty grid for heights up to 64")
    out = np.zeros_like(a)
    ref("2d_gpu").ref2d_gpu_thin_u8(w, h, _u8(a), _u8(out))
    return out


def ref_gpu_thin3d(vol: np.ndarray) -> np.ndarray:
    """The reference's own CUDA 3D library (dims multiples of 32, >= 64)."""
    a = np.ascontiguousarray(vol != 0, dtype=np.uint8)
    d, h, w = a.shape
    if any(n % 32 or n < 64 for n in (w, h, d)):
        raise ValueError("the reference 3D library needs dimensions that are multiples of 32 and >= 64")
    out = np.zeros_like(a)
    ref("3d_gpu").ref3d_gpu_thin_u8(w, h, d, _u8(a), _u8(out))
    return out


def ref_segments2d(img: np.ndarray) -> Segments:
    a = np.ascontiguousarray(img != 0, dtype=np.uint8)
    h, w = a.shape
    s = _Segs()
    ref("2d").ref2d_segments_u8(_u8(a), w, h, C.byref(s))
    return _take_segs(s, 2, ref("2d").ref_segs_free)


def ref_segments3d(vol: np.ndarray) -> Segments:
    a = np.ascontiguousarray(vol != 0, dtype=np.uint8)
    d, h, w = a.shape
    s = _Segs()
    ref("3d").ref3d_segments_u8(_u8(a), w, h, d, C.byref(s))
    return _take_segs(s, 3, ref("3d").ref_segs_free)


def _ref_cl_take(L, n, ox, oy, oz, oi) -> Centerline:
    npts = oi[n]
    out = Centerline(_arr(ox, npts, np.float32), _arr(oy, npts, np.float32),
                     _arr(oz, npts, np.float32) if oz is not None else None,
                     _arr(oi, n + 1, np.uint32))
    L.ref_free_f32(ox)
    L.ref_free_f32(oy)
    if oz is not None:
        L.ref_free_f32(oz)
    L.ref_free_u32(oi)
    return out


def ref_centerline2d(data: np.ndarray, dtype_code: int, max_segment_length: int,
                     smoothing_span: int) -> Centerline:
    a = np.ascontiguousarray(data)
    h, w = a.shape
    L = ref("2d")
    ox, oy = C.POINTER(C.c_float)(), C.POINTER(C.c_float)()
    oi = C.POINTER(C.c_uint32)()
    n = L.ref2d_centerline(dtype_code, a.ctypes.data_as(C.c_void_p), w, h, max_segment_length,
                           smoothing_span, C.byref(ox), C.byref(oy), C.byref(oi))
    return _ref_cl_take(L, n, ox, oy, None, oi)


def ref_centerline3d(data: np.ndarray, dtype_code: int, max_segment_length: int,
                     smoothing_span: int) -> Centerline:
    a = np.ascontiguousarray(data)
    d, h, w = a.shape
    L = ref("3d")
    ox, oy, oz = C.POINTER(C.c_float)(), C.POINTER(C.c_float)(), C.POINTER(C.c_float)()
    oi = C.POINTER(C.c_uint32)()
    n = L.ref3d_centerline(dtype_code, a.ctypes.data_as(C.c_void_p), w, h, d, max_segment_length,
                           smoothing_span, C.byref(ox), C.byref(oy), C.byref(oz), C.byref(oi))
    return _ref_cl_take(L, n, ox, oy, oz, oi)
