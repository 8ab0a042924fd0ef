"""ORACLE — test infrastructure. ctypes wrapper of oracle/cone_oracle.cpp.

Used only by tests/, __graft_entry__.smoke() and bench.py's CPU baseline, as
the checker of the CUDA library.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build import OUT, build

_lib = None

NODE_DTYPE = np.dtype([("lo", "<f4", 4), ("hi", "<f4", 4), ("info", "<u4", 4)])


class _Params(C.Structure):
    _fields_ = [("hierarchy", C.c_uint32), ("wide_extent", C.c_float), ("light_cone_cap", C.c_uint32),
                ("wide_cone_cap", C.c_uint32), ("prefilter", C.c_float), ("object_prefilter", C.c_uint32),
                ("accumulate", C.c_uint32), ("back_facing", C.c_uint32)]

#: How each mesh's cells are summed: the reference's sums in walk order in
#: the run's precision; each add rounded to 2^-24 of a bin into exact integer
#: cells (the CUDA library's accumulator); exact sums in double.
SUM_WALK_ORDER, SUM_FIXED, SUM_EXACT = 0, 1, 2


def load():
    global _lib
    if _lib is None:
        if not OUT.exists():
            build()
        lib = C.CDLL(str(OUT))
        P, U32, U64, I = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
        lib.oracle_scene_create.restype = P
        lib.oracle_scene_create.argtypes = [P, P, U32]
        lib.oracle_scene_destroy.argtypes = [P]
        lib.oracle_scene_sizes.argtypes = [P, P]
        lib.oracle_scene_arrays.argtypes = [P, P, P, P, P, P]
        lib.oracle_visibility.restype = I
        lib.oracle_visibility.argtypes = [P, P, U64, P, U32, C.POINTER(_Params), P, U64, I, P, P, P, P, P, P, P, I]
        lib.oracle_scene_coverage.argtypes = [P, P, P]
        lib.oracle_sky_visibility.restype = I
        lib.oracle_sky_visibility.argtypes = [P, P, U64, U32, U32, C.c_float, I, P, P, P, P, P, P, I, U32]
        lib.oracle_cpu_masked.restype = I
        lib.oracle_cpu_masked.argtypes = [P, P, U64, P, I, P, P, P, I]
        lib.oracle_disk_table.argtypes = [P]
        lib.oracle_cpu_masked_with.restype = I
        lib.oracle_cpu_masked_with.argtypes = [P, P, P, U64, P, P, P, P, I]
        lib.oracle_cpu_bvh_create.restype = P
        lib.oracle_cpu_bvh_create.argtypes = [P]
        lib.oracle_cpu_bvh_destroy.argtypes = [P]
        lib.oracle_primary_hits.argtypes = [P, P, U32, U32, P, P, I]
        lib.oracle_cpu_weights.restype = I
        lib.oracle_cpu_weights.argtypes = [P, P, P, P]
        lib.oracle_poly_overflows.restype = U64
        lib.oracle_scene_create_instanced.restype = P
        lib.oracle_scene_create_instanced.argtypes = [P, P, U32, P, U32, P, U32]
        lib.oracle_scene_move.argtypes = [P, P, P]
        lib.oracle_scene_set_clear.argtypes = [P, P, C.c_uint32]
        lib.oracle_stale_cones.argtypes = [P, P, U64, P, U32, P, U32, P, I]
        lib.oracle_scene_transforms.restype = U64
        lib.oracle_scene_transforms.argtypes = [P, P]
        _lib = lib
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def default_threads() -> int:
    return max(1, len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1))


class OracleScene:
    """The reference's host layouts built by the oracle's own restatement."""

    def __init__(self, meshes=None, tri9=None, counts=None):
        if meshes is not None:
            parts = [np.asarray(m, np.float32).reshape(-1, 9) for m in meshes]
            tri9 = np.concatenate(parts) if parts else np.zeros((0, 9), np.float32)
            counts = np.array([len(p) for p in parts], np.uint32)
        self.tri9 = np.ascontiguousarray(tri9, np.float32)
        self.counts = np.ascontiguousarray(counts, np.uint32)
        self._h = C.c_void_p(load().oracle_scene_create(_p(self.tri9), _p(self.counts), len(self.counts)))

    @classmethod
    def instanced(cls, geometries, instances: np.ndarray, movable=None) -> "OracleScene":
        """An instanced scene: geometries (object space) placed by cc_instance
        records (flatten_instanced, hierarchy.rs:464-522)."""
        self = cls.__new__(cls)
        parts = [np.asarray(m, np.float32).reshape(-1, 9) for m in geometries]
        self.tri9 = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros((0, 9), np.float32))
        self.counts = np.array([len(p) for p in parts], np.uint32)
        self.instances = np.ascontiguousarray(instances)
        self.movable = None if movable is None else np.ascontiguousarray(movable, np.uint32)
        self._h = C.c_void_p(load().oracle_scene_create_instanced(
            _p(self.tri9), _p(self.counts), len(self.counts), _p(self.instances), len(self.instances),
            _p(self.movable), 0 if self.movable is None else len(self.movable)))
        return self

    def set_clear(self, clear) -> None:
        """Each object's clear (Placement::clear, hierarchy.rs:266-270): 0 opaque,
        (0, 1) alpha-blended, below 0 transmissive (at most -2 a volume)."""
        c = np.ascontiguousarray(clear, np.float32)
        load().oracle_scene_set_clear(self._h, _p(c), len(c))

    def move(self, placements: np.ndarray) -> np.ndarray:
        """Places the movers anew (in their order); per mover its bounds before and after."""
        pl = np.ascontiguousarray(placements)
        boxes = np.zeros((len(pl), 12), np.float32)
        load().oracle_scene_move(self._h, _p(pl), _p(boxes))
        return boxes

    def stale_cones(self, receivers: np.ndarray, lights: np.ndarray, boxes: np.ndarray, threads=None) -> np.ndarray:
        rec = np.ascontiguousarray(receivers, np.float32).reshape(-1, 8)
        lig = np.ascontiguousarray(lights, np.float32).reshape(-1, 16)
        b = np.ascontiguousarray(boxes, np.float32).reshape(-1, 12)
        out = np.zeros(rec.shape[0] * lig.shape[0], np.uint8)
        load().oracle_stale_cones(self._h, _p(rec), rec.shape[0], _p(lig), lig.shape[0], _p(b), b.shape[0], _p(out),
                                  int(threads or default_threads()))
        return out

    def transforms(self) -> np.ndarray:
        n = int(load().oracle_scene_transforms(self._h, None))
        out = np.zeros((n, 16), np.float32)
        if n:
            load().oracle_scene_transforms(self._h, _p(out))
        return out

    def sizes(self) -> dict:
        out = np.zeros(6, np.uint64)
        load().oracle_scene_sizes(self._h, _p(out))
        keys = ("ntris", "nmeshes", "nblas", "nblas_items", "nnodes", "nitems")
        return {k: int(v) for k, v in zip(keys, out)}

    def arrays(self) -> dict:
        sz = self.sizes()
        ranges = np.zeros((sz["nmeshes"], 4), np.uint32)
        blas = np.zeros(sz["nblas"], NODE_DTYPE)
        blas_items = np.zeros(sz["nblas_items"], np.uint32)
        nodes = np.zeros(sz["nnodes"], NODE_DTYPE)
        items = np.zeros(sz["nitems"], np.uint32)
        load().oracle_scene_arrays(self._h, _p(ranges), _p(blas), _p(blas_items), _p(nodes), _p(items))
        return dict(ranges=ranges, blas=blas, blas_items=blas_items, nodes=nodes, items=items)

    def visibility(self, receivers: np.ndarray, lights: np.ndarray, hierarchy: int = 2, precision: int = 4,
                   cone_ids: np.ndarray | None = None, threads: int | None = None, wide_extent: float = 8.0,
                   light_cone_cap: int = 4096, wide_cone_cap: int = 512, partial: bool = True, prefilter: float = 0.0,
                   object_prefilter: bool = True, accumulate: int = 0, back_facing: bool = False) -> dict:
        """Per-cone results (cone c = light * npoints + point), for all cones or
        the `cone_ids` subset (outputs in subset order)."""
        rec = np.ascontiguousarray(receivers, np.float32).reshape(-1, 8)
        lig = np.ascontiguousarray(lights, np.float32).reshape(-1, 16)
        n = rec.shape[0] * lig.shape[0] if cone_ids is None else len(cone_ids)
        ids = None if cone_ids is None else np.ascontiguousarray(cone_ids, np.uint64)
        full = np.zeros((n, 2), np.uint32)
        any_ = np.zeros((n, 2), np.uint32)
        part = np.zeros((n, 64), np.float32) if partial else None
        irr = np.zeros(n, np.float32)
        frac = np.zeros(n, np.float32)
        work = np.zeros((n, 4), np.uint32)
        unsh = np.zeros(n, np.float32)
        prm = _Params(hierarchy, wide_extent, light_cone_cap, wide_cone_cap, prefilter, 1 if object_prefilter else 0,
                      int(accumulate), 1 if back_facing else 0)
        rc = load().oracle_visibility(self._h, _p(rec), rec.shape[0], _p(lig), lig.shape[0], C.byref(prm), _p(ids),
                                      0 if ids is None else len(ids), precision, _p(full), _p(any_), _p(part),
                                      _p(irr), _p(frac), _p(work), _p(unsh), threads or default_threads())
        if rc != 0:
            raise RuntimeError(f"oracle_visibility failed: {rc}")
        return dict(full=full.view(np.uint64).reshape(n), any=any_.view(np.uint64).reshape(n), partial=part,
                    irradiance=irr, fraction=frac, work=work, unshadowed=unsh)

    def coverage(self) -> tuple:
        """(triangle-hierarchy nodes' samples (n, 27), object nodes' (m, 27) or None)."""
        sizes = self.sizes()
        blas = np.zeros((sizes["nblas"], 27), np.float32)
        obj = np.zeros((sizes["nnodes"], 27), np.float32) if getattr(self, "instances", None) is not None else None
        load().oracle_scene_coverage(self._h, _p(blas), _p(obj))
        return blas, obj

    def sky_visibility(self, receivers: np.ndarray, hierarchy: int = 2, flags: int = 0, precision: int = 4,
                       threads: int | None = None, faces: bool = True, prefilter: float = 0.0,
                       accumulate: int = 0) -> dict:
        """Sky cones (six cube faces per receiver): irradiance per unit sky
        radiance per receiver, and per face cone c = face * npoints + point its
        light, FULL/ANY words, coverage and work counters. flags: 1 combine
        meshes by the maximum, 2 walk geometry below the horizon too, 8 faces
        in the frame of the object each receiver lies on (its point.w holds
        the object's index as the bits of a uint32)."""
        rec = np.ascontiguousarray(receivers, np.float32).reshape(-1, 8)
        n = rec.shape[0]
        irr = np.zeros(n, np.float32)
        out = dict(irradiance=irr)
        if faces:
            out.update(face_light=np.zeros(6 * n, np.float32), full=np.zeros((6 * n, 2), np.uint32),
                       any=np.zeros((6 * n, 2), np.uint32), partial=np.zeros((6 * n, 64), np.float32),
                       work=np.zeros((6 * n, 4), np.uint32))
        g = out.get
        rc = load().oracle_sky_visibility(self._h, _p(rec), n, hierarchy, flags, prefilter, precision, _p(irr),
                                          _p(g("face_light")),
                                          _p(g("full")), _p(g("any")), _p(g("partial")), _p(g("work")),
                                          threads or default_threads(), int(accumulate))
        if rc != 0:
            raise RuntimeError(f"oracle_sky_visibility failed: {rc}")
        if faces:
            out["full"] = out["full"].view(np.uint64).reshape(6 * n)
            out["any"] = out["any"].view(np.uint64).reshape(6 * n)
        return out

    def cpu_masked(self, receivers: np.ndarray, light9, use_bvh: bool = False, threads: int | None = None):
        """The reference CPU path (cone3 + coverage, Receiver::masked): (visible, total weight)."""
        rec = np.ascontiguousarray(receivers, np.float32).reshape(-1, 8)
        l9 = np.ascontiguousarray(light9, np.float32).reshape(9)
        vis = np.zeros(rec.shape[0], np.float32)
        tot = np.zeros(rec.shape[0], np.float32)
        visited = np.zeros(rec.shape[0], np.uint32)
        load().oracle_cpu_masked(self._h, _p(rec), rec.shape[0], _p(l9), int(use_bvh), _p(vis), _p(tot),
                                 _p(visited), threads or default_threads())
        return vis, tot

    def cpu_bvh(self) -> "CpuBvh":
        """The reference CPU path's leaf-4 BVH (bvh.rs), built alone so that
        its build time can be measured apart from the cones."""
        return CpuBvh(self)

    def cpu_masked_with(self, bvh: "CpuBvh | None", receivers: np.ndarray, light9, threads: int | None = None):
        """cpu_masked over a prebuilt BVH (None: every triangle tested)."""
        rec = np.ascontiguousarray(receivers, np.float32).reshape(-1, 8)
        l9 = np.ascontiguousarray(light9, np.float32).reshape(9)
        vis = np.zeros(rec.shape[0], np.float32)
        tot = np.zeros(rec.shape[0], np.float32)
        load().oracle_cpu_masked_with(self._h, None if bvh is None else bvh._h, _p(rec), rec.shape[0], _p(l9),
                                      _p(vis), _p(tot), None, threads or default_threads())
        return vis, tot

    def primary_hits(self, camera, width: int, height: int, threads: int | None = None):
        """Receivers (H*W, 8) at a pinhole camera's primary hits and the hit
        mask, cast over this scene's own hierarchies (the same receivers as
        the library's host caster, bit for bit)."""
        cam = np.ascontiguousarray(np.asarray(camera, np.float32).reshape(10))
        out = np.zeros((width * height, 8), np.float32)
        hit = np.zeros(width * height, np.uint8)
        load().oracle_primary_hits(self._h, _p(cam), int(width), int(height), _p(out), _p(hit),
                                   int(threads or default_threads()))
        return out, hit

    def close(self):
        if self._h:
            load().oracle_scene_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CpuBvh:
    """The reference CPU path's BVH over an OracleScene's triangles."""

    def __init__(self, scene: OracleScene):
        self.scene = scene
        self._h = C.c_void_p(load().oracle_cpu_bvh_create(scene._h))

    def close(self):
        if self._h:
            load().oracle_cpu_bvh_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def disk_table() -> np.ndarray:
    out = np.zeros(64, np.float64)
    load().oracle_disk_table(_p(out))
    return out


def cpu_weights(point, normal, light9) -> np.ndarray:
    p = np.ascontiguousarray(point, np.float32)
    n = np.ascontiguousarray(normal, np.float32)
    l9 = np.ascontiguousarray(light9, np.float32)
    w = np.zeros(64, np.float32)
    if load().oracle_cpu_weights(_p(p), _p(n), _p(l9), _p(w)) != 0:
        raise ValueError("no cone")
    return w


def poly_overflows() -> int:
    return int(load().oracle_poly_overflows())
