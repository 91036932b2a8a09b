"""Loader for the native library ``libbgt.so`` (ctypes over the C ABI in
``include/bgt_capi.h``).  There is no fallback: if the library cannot be
loaded, every entry point raises."""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libbgt.so")
SYNTH_PATH = os.path.join(PKG, "libbgt_synth.so")

# names declared in include/bgt_capi.h (kept in sync by tests/test_capi_symbols.py)
EXPORTS = [
    "bgt_ctx_create", "bgt_ctx_destroy", "bgt_ctx_set_stream", "bgt_last_error", "bgt_version",
    "bgt_thin2d", "bgt_thin3d", "bgt_thin2d_device", "bgt_thin3d_device", "bgt_thin2d_device_noalloc",
    "bgt_centerline2d", "bgt_centerline3d", "bgt_free", "bgt_matlab_segments",
    "bgt_segments2d_device", "bgt_segments3d_device",
    "bgt_batch_create", "bgt_batch_destroy", "bgt_batch_add2d", "bgt_batch_add3d", "bgt_batch_finalize",
    "bgt_batch_reserve", "bgt_batch_reset", "bgt_batch_set_grid",
    "bgt_batch_set_io", "bgt_batch_run", "bgt_batch_instance_stats", "bgt_batch_device_bytes", "bgt_batch_work", "bgt_batch_stage_ms",
    "bgt_batch_engine_ms", "bgt_batch_set_engine", "bgt_batch_plan", "bgt_batch_res_trace",
    "bgt_tune_class", "bgt_tune_set", "bgt_tune_get", "bgt_cfg_list", "bgt_cfg_describe", "bgt_rule_table",
    "bgt_server_create", "bgt_server_submit", "bgt_server_poll", "bgt_server_drain", "bgt_server_stats",
    "bgt_server_reset_stats", "bgt_server_destroy", "bgt_server_memory",
]


class BGTError(RuntimeError):
    """A C-ABI call returned a nonzero bgt_status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"bgt error {code}: {msg}")
        self.code = code


_lib = None
_synth = None

P = C.c_void_p
I = C.c_int
PP = C.POINTER(C.c_void_p)


def _declare(L):
    vp, ip, up = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_uint)
    fpp = C.POINTER(C.POINTER(C.c_float))
    upp = C.POINTER(C.POINTER(C.c_uint))
    sig = {
        "bgt_ctx_create": [I, C.POINTER(vp)],
        "bgt_ctx_destroy": [vp],
        "bgt_ctx_set_stream": [vp, vp],
        "bgt_version": [],
        "bgt_thin2d": [vp, I, vp, I, I, vp],
        "bgt_thin3d": [vp, I, vp, I, I, I, vp],
        "bgt_thin2d_device": [vp, I, vp, I, I, vp],
        "bgt_thin3d_device": [vp, I, vp, I, I, I, vp],
        "bgt_thin2d_device_noalloc": [I, I, vp, I, I, vp, vp],
        "bgt_centerline2d": [vp, I, vp, I, I, I, I, fpp, fpp, upp, up],
        "bgt_centerline3d": [vp, I, vp, I, I, I, I, I, fpp, fpp, fpp, upp, up],
        "bgt_segments2d_device": [vp, I, vp, I, I, C.POINTER(C.POINTER(C.c_int32)),
                                  C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.POINTER(C.c_int16)),
                                  C.POINTER(C.POINTER(C.c_int16)), ip, ip],
        "bgt_segments3d_device": [vp, I, vp, I, I, I, C.POINTER(C.POINTER(C.c_int32)),
                                  C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.POINTER(C.c_int16)),
                                  C.POINTER(C.POINTER(C.c_int16)), C.POINTER(C.POINTER(C.c_int16)), ip, ip],
        "bgt_batch_create": [vp, C.POINTER(vp)],
        "bgt_batch_destroy": [vp],
        "bgt_batch_add2d": [vp, I, I, I, ip],
        "bgt_batch_add3d": [vp, I, I, I, I, ip],
        "bgt_batch_finalize": [vp],
        "bgt_batch_reserve": [vp, C.c_size_t],
        "bgt_batch_reset": [vp],
        "bgt_batch_set_grid": [vp, I],
        "bgt_batch_set_io": [vp, I, I, vp, vp],
        "bgt_batch_run": [vp, I, I],
        "bgt_batch_instance_stats": [vp, I, ip, ip, ip],
        "bgt_batch_device_bytes": [vp, C.POINTER(C.c_size_t)],
        "bgt_batch_work": [vp, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)],
        "bgt_batch_stage_ms": [vp, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)],
        "bgt_batch_engine_ms": [vp, C.POINTER(C.c_float), C.POINTER(C.c_float)],
        "bgt_batch_set_engine": [vp, I],
        "bgt_batch_plan": [vp, I, ip, ip],
        "bgt_batch_res_trace": [vp, ip, ip, ip, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), ip, I],
        "bgt_tune_class": [I, I, I, I],
        "bgt_tune_set": [I, I, I],
        "bgt_tune_get": [I, I, ip],
        "bgt_cfg_list": [I, ip, I, ip],
        "bgt_cfg_describe": [I, ip, ip, ip, ip, ip, ip],
        "bgt_matlab_segments": [I, C.c_uint, vp, vp, vp, vp, vp],
        "bgt_rule_table": [I, I, vp, vp],
        "bgt_server_create": [I, C.c_size_t, C.POINTER(vp)],
        "bgt_server_submit": [vp, I, vp, I, I, I, vp, C.POINTER(C.c_ulonglong)],
        "bgt_server_poll": [vp, C.POINTER(C.c_ulonglong), C.POINTER(C.c_double), ip, I, ip],
        "bgt_server_drain": [vp, C.c_double],
        "bgt_server_stats": [vp, I, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                             C.POINTER(C.c_ulonglong)],
        "bgt_server_reset_stats": [vp],
        "bgt_server_memory": [vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.POINTER(C.c_ulonglong)],
        "bgt_server_destroy": [vp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.bgt_last_error.argtypes = []
    L.bgt_last_error.restype = C.c_char_p
    L.bgt_free.argtypes = [vp]
    L.bgt_free.restype = None


def lib():
    """The loaded libbgt.so (raises if it is missing: there is no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"native library {LIB_PATH} not built; run python -m begputhinning_b200.build")
        L = C.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != 0:
        raise BGTError(rc, lib().bgt_last_error().decode(errors="replace"))


def synth():
    global _synth
    if _synth is None:
        if not os.path.exists(SYNTH_PATH):
            raise ImportError(f"{SYNTH_PATH} not built; run python -m begputhinning_b200.build")
        L = C.CDLL(SYNTH_PATH)
        u8p = C.POINTER(C.c_uint8)
        dp = C.POINTER(C.c_double)
        d = C.c_double
        L.bgt_synth_uniform.argtypes = [C.c_uint64, C.c_int64, dp]
        L.bgt_synth_render_strokes2d.argtypes = [I, I, I, dp, dp, u8p]
        L.bgt_synth_strokes2d.argtypes = [C.c_uint64, I, I, I, d, d, u8p]
        L.bgt_synth_vessels2d.argtypes = [C.c_uint64, I, I, I, I, d, d, d, d, d, d, d, I, d, d, u8p]
        L.bgt_synth_trees3d.argtypes = [C.c_uint64, I, I, I, I, I, d, d, d, d, d, d, I, d, d, u8p]
        for n in ["bgt_synth_uniform", "bgt_synth_render_strokes2d", "bgt_synth_strokes2d",
                  "bgt_synth_vessels2d", "bgt_synth_trees3d"]:
            getattr(L, n).restype = None
        _synth = L
    return _synth
