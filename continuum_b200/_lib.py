"""ctypes binding of libcontinuum_cuda.so (include/continuum_cuda.h).

The library is built in-tree by ``python -m continuum_b200.build``; loading
fails loudly if it is missing. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libcontinuum_cuda.so"

CC_OK = 0
CC_ERR_INVALID = 1
CC_ERR_CUDA = 2
CC_ERR_OOM = 3
CC_ERR_NO_DEVICE = 4
CC_ERR_STACK = 5
CC_ERR_TIMEOUT = 6
CC_ERR_BUSY = 7
CC_NONE = 0xFFFFFFFF

CC_DEVICE_POINTERS = 1
CC_NO_REDO = 2
CC_KEEP_ORDER = 4
CC_STATIC_MAX_CONES = 131072
CC_BATCH_GRAPH = 8

CC_CONE_CAPPED = 1
CC_CONE_STACK = 2
CC_CONE_DIVERGED = 4
CC_CONE_REWALKED = 8
CC_CONE_FULL_STOP = 16
CC_CONE_ACC_WIDE = 32
CC_NO_OBJECT_PREFILTER = 8
CC_BACK_FACING = 16
CC_SKY_COMBINE_MAX = 1
CC_SKY_NO_HORIZON_CULL = 2
CC_SKY_OBJECT_FRAME = 4

#: Every symbol include/continuum_cuda.h declares.
EXPORTS = (
    "cc_context_create", "cc_context_destroy", "cc_context_set_split_chunk", "cc_last_error", "cc_scene_upload", "cc_scene_build",
    "cc_scene_destroy", "cc_scene_sizes", "cc_scene_arrays", "cc_scene_device_bytes", "cc_options_default",
    "cc_visibility", "cc_irradiance", "cc_coverage", "cc_scene_primary_hits", "cc_context_kernel_times",
    "cc_visibility_static", "cc_batch_options_default", "cc_batch_create", "cc_batch_destroy", "cc_batch_clear",
    "cc_batch_add", "cc_batch_add_update", "cc_batch_submit", "cc_batch_wait", "cc_batch_tune", "cc_batch_sizes",
    "cc_server_options_default", "cc_server_create", "cc_server_destroy", "cc_server_add_scene", "cc_server_submit",
    "cc_server_wait", "cc_server_stats", "cc_scene_build_instanced", "cc_scene_transforms", "cc_scene_move", "cc_scene_set_clear",
    "cc_stale_cones", "cc_visibility_update", "cc_cache_options_default", "cc_cache_create", "cc_cache_destroy",
    "cc_cache_frame", "cc_cache_read", "cc_cache_pool", "cc_cache_jobs", "cc_planner_create", "cc_planner_destroy",
    "cc_planner_frame", "cc_planner_jobs", "cc_planner_slot", "cc_sky_visibility", "cc_scene_coverage",
)

# cc_instance: an object placing a geometry (world = scale * rotation * p + translation).
INSTANCE_DTYPE = np.dtype([("geometry", "<u4"), ("rotation", "<f4", 9), ("scale", "<f4"), ("translation", "<f4", 3)])


class CCError(RuntimeError):
    """A non-zero status from the library, with its message."""

    def __init__(self, code: int, message: str):
        super().__init__(f"continuum_cuda error {code}: {message}")
        self.code = code


class FlatScene(C.Structure):
    _fields_ = [
        ("tris", C.c_void_p), ("ntris", C.c_uint32),
        ("ranges", C.c_void_p), ("nmeshes", C.c_uint32),
        ("blas", C.c_void_p), ("nblas", C.c_uint32),
        ("blas_items", C.c_void_p), ("nblas_items", C.c_uint32),
        ("nodes", C.c_void_p), ("nnodes", C.c_uint32),
        ("items", C.c_void_p), ("nitems", C.c_uint32),
        ("xforms", C.c_void_p), ("nxforms", C.c_uint32),
    ]


class Options(C.Structure):
    _fields_ = [
        ("hierarchy", C.c_uint32), ("wide_extent", C.c_float), ("light_cone_cap", C.c_uint32),
        ("wide_cone_cap", C.c_uint32), ("points_per_warp", C.c_uint32), ("flags", C.c_uint32),
        ("prefilter", C.c_float),
    ]


class BatchOptions(C.Structure):
    _fields_ = [("points_per_warp", C.c_uint32), ("blocks_per_sm", C.c_uint32), ("flags", C.c_uint32)]


class ServerOptions(C.Structure):
    _fields_ = [("hbm_budget", C.c_uint64), ("max_inflight", C.c_uint32), ("max_queue", C.c_uint32),
                ("max_launch_cones", C.c_uint64), ("points_per_warp", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("deadline_ns_per_cone", C.c_uint32)]


class CacheOptions(C.Structure):
    _fields_ = [("pages", C.c_uint32), ("bake_budget", C.c_uint32), ("frame_target_ms", C.c_float),
                ("frame_budget_ms", C.c_float), ("floor_overrun", C.c_float), ("light_ratio", C.c_uint32)]


class PageRequest(C.Structure):
    _fields_ = [("key", C.c_uint32 * 3), ("priority", C.c_uint32), ("inside", C.c_uint32 * 2), ("texels", C.c_void_p)]


class CacheFrameInfo(C.Structure):
    _fields_ = [("period_ms", C.c_float), ("render_ms", C.c_float), ("gpu_waited", C.c_uint32)]


class CacheStats(C.Structure):
    _fields_ = [("budget", C.c_float), ("frame", C.c_uint32), ("pages_planned", C.c_uint32), ("jobs", C.c_uint32),
                ("spent", C.c_uint32), ("resident", C.c_uint32), ("evicted", C.c_uint32), ("last_bake_ms", C.c_float)]


class Request(C.Structure):
    _fields_ = [("scene", C.c_uint32), ("receivers", C.c_void_p), ("npoints", C.c_uint64), ("lights", C.c_void_p),
                ("nlights", C.c_uint32), ("hierarchy", C.c_uint32), ("cache_key", C.c_uint64),
                ("full", C.c_void_p), ("any", C.c_void_p), ("irradiance", C.c_void_p), ("fraction", C.c_void_p),
                ("prefilter", C.c_float)]


class RequestStats(C.Structure):
    _fields_ = [("queued_ms", C.c_double), ("total_ms", C.c_double), ("launch_requests", C.c_uint32),
                ("cached_lights", C.c_uint32)]


class Outputs(C.Structure):
    _fields_ = [
        ("full", C.c_void_p), ("any", C.c_void_p), ("partial", C.c_void_p),
        ("irradiance", C.c_void_p), ("fraction", C.c_void_p), ("work", C.c_void_p),
    ]


_lib: C.CDLL | None = None


def load() -> C.CDLL:
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m continuum_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    P, U32, U64, I = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
    sig = {
        "cc_context_create": (I, [I, C.POINTER(P)]),
        "cc_context_destroy": (I, [P]),
        "cc_context_set_split_chunk": (I, [P, C.c_uint64]),
        "cc_last_error": (C.c_char_p, []),
        "cc_scene_upload": (I, [P, C.POINTER(FlatScene), C.POINTER(P)]),
        "cc_scene_build": (I, [P, P, P, U32, C.POINTER(P)]),
        "cc_scene_destroy": (I, [P]),
        "cc_scene_sizes": (I, [P, P]),
        "cc_scene_arrays": (I, [P, P, P, P, P, P]),
        "cc_scene_device_bytes": (U64, [P]),
        "cc_options_default": (None, [C.POINTER(Options)]),
        "cc_visibility": (I, [P, P, P, U64, P, U32, C.POINTER(Options), C.POINTER(Outputs), P]),
        "cc_irradiance": (I, [P, P, U64, P, I, P, P, U32, U32, U32, P, C.POINTER(C.c_double)]),
        "cc_coverage": (I, [P, P, U64, P, I, P, P, U32, P]),
        "cc_scene_primary_hits": (I, [P, P, U32, U32, P, P]),
        "cc_context_kernel_times": (I, [P, P, I]),
        "cc_visibility_static": (I, [P, P, U64, P, U32, C.POINTER(Options), C.POINTER(Outputs), P]),
        "cc_batch_options_default": (None, [C.POINTER(BatchOptions)]),
        "cc_batch_create": (I, [P, C.POINTER(P)]),
        "cc_batch_destroy": (I, [P]),
        "cc_batch_clear": (I, [P]),
        "cc_batch_add": (I, [P, P, P, U64, P, U32, C.POINTER(Options), C.POINTER(Outputs), C.POINTER(U32)]),
        "cc_batch_add_update": (I, [P, P, P, U64, P, U32, P, C.POINTER(Options), C.POINTER(Outputs), C.POINTER(U32)]),
        "cc_batch_submit": (I, [P, C.POINTER(BatchOptions), P]),
        "cc_batch_wait": (I, [P, U32]),
        "cc_batch_tune": (I, [P, C.POINTER(BatchOptions), U32, C.POINTER(BatchOptions), P, U32]),
        "cc_batch_sizes": (I, [P, P]),
        "cc_server_options_default": (None, [C.POINTER(ServerOptions)]),
        "cc_server_create": (I, [P, C.POINTER(ServerOptions), C.POINTER(P)]),
        "cc_server_destroy": (I, [P]),
        "cc_server_add_scene": (I, [P, P, C.POINTER(U32)]),
        "cc_server_submit": (I, [P, C.POINTER(Request), C.POINTER(U64)]),
        "cc_server_wait": (I, [P, U64, U32, C.POINTER(RequestStats)]),
        "cc_server_stats": (I, [P, P]),
        "cc_scene_build_instanced": (I, [P, P, P, U32, P, U32, P, U32, C.POINTER(P)]),
        "cc_scene_move": (I, [P, P, U32, P]),
        "cc_scene_set_clear": (I, [P, P, U32]),
        "cc_stale_cones": (I, [P, P, P, U64, P, U32, P, U32, P, C.POINTER(U64), P]),
        "cc_visibility_update": (I, [P, P, P, U64, P, U32, P, C.POINTER(Options), C.POINTER(Outputs), C.POINTER(U64), P]),
        "cc_scene_transforms": (U64, [P, P, U64]),
        "cc_cache_options_default": (None, [C.POINTER(CacheOptions)]),
        "cc_cache_create": (I, [P, P, P, U32, C.POINTER(CacheOptions), C.POINTER(P)]),
        "cc_cache_destroy": (I, [P]),
        "cc_cache_frame": (I, [P, P, U32, C.POINTER(CacheFrameInfo), C.POINTER(CacheStats)]),
        "cc_cache_read": (I, [P, P, P]),
        "cc_cache_pool": (I, [P, C.POINTER(P), C.POINTER(U32)]),
        "cc_cache_jobs": (C.c_int64, [P, P, U64, P, U32]),
        "cc_planner_create": (I, [C.POINTER(CacheOptions), U32, C.POINTER(P)]),
        "cc_planner_destroy": (I, [P]),
        "cc_planner_frame": (I, [P, P, U32, C.POINTER(CacheFrameInfo), C.c_float, C.POINTER(CacheStats)]),
        "cc_planner_jobs": (C.c_int64, [P, P, U64, P, U32]),
        "cc_planner_slot": (C.c_int64, [P, P]),
        "cc_sky_visibility": (I, [P, P, P, U64, C.POINTER(Options), U32, P, C.POINTER(Outputs), P]),
        "cc_scene_coverage": (C.c_int64, [P, P, U64, P, U64]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(code: int) -> None:
    if code != CC_OK:
        msg = load().cc_last_error()
        raise CCError(code, msg.decode() if msg else "")


def ptr(a: np.ndarray | None) -> int | None:
    """Host address of a C-contiguous array (None for None)."""
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data


def default_options() -> Options:
    o = Options()
    load().cc_options_default(C.byref(o))
    return o
