"""The reference-facing visibility API over the CUDA library.

Mirrors ``continuum_gpu::MaskConeKernel`` (crates/continuum-gpu/src/lib.rs:65-120)
for the mask-cone light path: ``irradiance`` / ``irradiance_with``
(lib.rs:1706-1730), ``coverage`` (lib.rs:3289-3298) and the light types
``RectLight`` / ``Light`` / ``SphereLight`` / ``Spot`` (lib.rs:552-609), plus
resident scenes and the multi-light ``visibility`` call with FULL/ANY mask
words, per-bin coverage and visible fractions.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from enum import IntEnum
from typing import Iterable, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import CCError, check, load, ptr


class Hierarchy(IntEnum):
    """How far cones descend before testing triangles (hierarchy.rs:731-749)."""

    NONE = 0
    MESHES = 1
    TRIANGLES = 2

    @staticmethod
    def of(x) -> "Hierarchy":
        if isinstance(x, bool):  # impl From<bool> for Hierarchy (hierarchy.rs:751-760)
            return Hierarchy.TRIANGLES if x else Hierarchy.NONE
        return Hierarchy(int(x))


def _v3(v) -> np.ndarray:
    a = np.asarray(v, dtype=np.float32).reshape(3)
    return a


@dataclass(frozen=True)
class RectLight:
    """A rectangular light: a corner and two perpendicular edges (lib.rs:552-566)."""

    corner: Sequence[float]
    edge_u: Sequence[float]
    edge_v: Sequence[float]
    one_sided: bool = False


@dataclass(frozen=True)
class Spot:
    """A spot's cone as glTF's: half-angles in radians (lib.rs:588-599)."""

    axis: Sequence[float]
    inner: float
    outer: float


@dataclass(frozen=True)
class SphereLight:
    """A spherical light seen from outside as a disk (lib.rs:576-586)."""

    center: Sequence[float]
    radius: float
    spot: Optional[Spot] = None


@dataclass(frozen=True)
class Light:
    """A light and its RGB radiance (lib.rs:568-574)."""

    emitter: object
    radiance: Sequence[float] = (1.0, 1.0, 1.0)

    @staticmethod
    def rect(rect: RectLight, radiance=(1.0, 1.0, 1.0)) -> "Light":
        return Light(rect, tuple(radiance))

    @staticmethod
    def white(rect: RectLight, radiance: float) -> "Light":
        return Light(rect, (radiance,) * 3)

    @staticmethod
    def point(center, radius: float, intensity=(1.0, 1.0, 1.0)) -> "Light":
        rad = tuple(float(i) / (math.pi * radius * radius) for i in intensity)
        return Light(SphereLight(tuple(center), float(radius)), rad)

    @staticmethod
    def spot(center, radius: float, intensity, spot: Spot) -> "Light":
        base = Light.point(center, radius, intensity)
        return Light(SphereLight(tuple(center), float(radius), spot), base.radiance)

    def as_rect(self) -> Optional[RectLight]:
        return self.emitter if isinstance(self.emitter, RectLight) else None


def light_gpu(light) -> np.ndarray:
    """The 16-float record the kernels read (LightGpu, lib.rs:710-749)."""
    if isinstance(light, RectLight):
        light = Light(light)
    out = np.zeros(16, dtype=np.float32)
    out[12:15] = np.asarray(light.radiance, dtype=np.float32)
    e = light.emitter
    if isinstance(e, RectLight):
        out[0:3] = _v3(e.corner)
        out[3] = 1.0 if e.one_sided else 0.0
        out[4:7] = _v3(e.edge_u)
        out[8:11] = _v3(e.edge_v)
    elif isinstance(e, SphereLight):
        out[0:3] = _v3(e.center)
        out[3] = 2.0
        if e.spot is not None:
            scale = 1.0 / max(math.cos(e.spot.inner) - math.cos(e.spot.outer), 1e-3)
            axis = np.asarray(e.spot.axis, dtype=np.float64)
            axis = axis / np.linalg.norm(axis)
            out[4:7] = (e.radius, scale, -math.cos(e.spot.outer) * scale)
            out[8:11] = axis
            out[11] = 1.0
        else:
            out[4:7] = (e.radius, 0.0, 1.0)
            out[8:11] = (0.0, 0.0, 1.0)
    else:
        raise TypeError(f"not a light: {light!r}")
    return out


def lights_gpu(lights: Iterable) -> np.ndarray:
    return np.stack([light_gpu(l) for l in lights]).astype(np.float32)


def receivers_gpu(receivers) -> np.ndarray:
    """(N, 8) float32 from (point, normal) pairs given as (N, 2, 3) or (N, 6)."""
    r = np.asarray(receivers, dtype=np.float32)
    if r.ndim == 2 and r.shape[1] == 8:
        return np.ascontiguousarray(r)
    r = r.reshape(-1, 6)
    out = np.zeros((r.shape[0], 8), dtype=np.float32)
    out[:, 0:3] = r[:, 0:3]
    out[:, 4:7] = r[:, 3:6]
    return out


def flatten_meshes(meshes) -> tuple[np.ndarray, np.ndarray]:
    """(tri9 float32 [T, 9], counts uint32 [M]) from a list of (n, 3, 3) arrays."""
    parts, counts = [], []
    for m in meshes:
        a = np.asarray(m, dtype=np.float32).reshape(-1, 9)
        parts.append(a)
        counts.append(a.shape[0])
    tri9 = np.concatenate(parts) if parts else np.zeros((0, 9), np.float32)
    return np.ascontiguousarray(tri9, dtype=np.float32), np.asarray(counts, dtype=np.uint32)


NODE_DTYPE = np.dtype([("lo", "<f4", 4), ("hi", "<f4", 4), ("info", "<u4", 4)])


@dataclass
class Visibility:
    """Per-cone results, shaped [lights, points]."""

    full: Optional[np.ndarray] = None        # uint64 mask words: bins wholly covered
    any: Optional[np.ndarray] = None         # uint64 mask words: bins with coverage > 0
    partial: Optional[np.ndarray] = None     # float32 [..., 64] per-bin coverage
    irradiance: Optional[np.ndarray] = None  # float32 irradiance per unit radiance
    fraction: Optional[np.ndarray] = None    # float32 visible fraction of the unshadowed light
    work: Optional[np.ndarray] = None        # uint32 [..., 4]: object nodes, triangle nodes, triangles, status


class Scene:
    """A scene resident on the device: triangles and both hierarchy levels."""

    def __init__(self, kernel: "MaskConeKernel", handle: int):
        self._kernel = kernel
        self._h = C.c_void_p(handle)

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise ValueError("scene is closed")
        return self._h

    def sizes(self) -> dict:
        out = np.zeros(6, dtype=np.uint64)
        check(load().cc_scene_sizes(self.handle, ptr(out)))
        keys = ("ntris", "nmeshes", "nblas", "nblas_items", "nnodes", "nitems")
        return {k: int(v) for k, v in zip(keys, out)}

    def coverage(self) -> tuple:
        """The prefiltered cones' coverage samples: (triangle-hierarchy nodes
        (n, 27), object nodes (m, 27) for an instanced scene, else None)."""
        sz = self.sizes()
        blas = np.zeros((max(sz["nblas"], 1), 27), np.float32)
        inst = self.transforms().shape[0] > 0
        obj = np.zeros((max(sz["nnodes"], 1), 27), np.float32) if inst else None
        n = load().cc_scene_coverage(self.handle, ptr(blas), sz["nblas"], ptr(obj), sz["nnodes"] if inst else 0)
        if n < 0:
            check(int(-n))
        return blas[: sz["nblas"]], (obj[: sz["nnodes"]] if inst else None)

    def arrays(self) -> dict:
        """The host layouts (hierarchy.rs Flat + mesh_hierarchy), for checking the builder."""
        sz = self.sizes()
        ranges = np.zeros((sz["nmeshes"], 4), np.uint32)
        blas = np.zeros(sz["nblas"], NODE_DTYPE)
        blas_items = np.zeros(sz["nblas_items"], np.uint32)
        nodes = np.zeros(sz["nnodes"], NODE_DTYPE)
        items = np.zeros(sz["nitems"], np.uint32)
        check(load().cc_scene_arrays(self.handle, ptr(ranges), ptr(blas), ptr(blas_items), ptr(nodes), ptr(items)))
        return dict(ranges=ranges, blas=blas, blas_items=blas_items, nodes=nodes, items=items)

    def move(self, placements) -> np.ndarray:
        """Places the movable objects anew (in their order); returns per mover
        its padded world bounds before and after (12 floats)."""
        inst = instances_array(placements)
        boxes = np.zeros((len(inst), 12), np.float32)
        check(load().cc_scene_move(self.handle, ptr(inst), len(inst), ptr(boxes)))
        return boxes

    def set_clear(self, clear) -> None:
        """Each object's `clear` (cc_scene_set_clear): 0 opaque, (0, 1)
        alpha-blended, below 0 transmissive (at most -2 a volume)."""
        c = np.ascontiguousarray(clear, np.float32)
        check(load().cc_scene_set_clear(self.handle, ptr(c), len(c)))

    def transforms(self) -> np.ndarray:
        """The objects' transforms, 16 floats each (instanced scenes; else empty)."""
        n = int(load().cc_scene_transforms(self.handle, None, 0))
        out = np.zeros((n, 16), np.float32)
        if n:
            load().cc_scene_transforms(self.handle, ptr(out), n)
        return out

    @property
    def device_bytes(self) -> int:
        return int(load().cc_scene_device_bytes(self.handle))

    def primary_hits(self, camera, width: int, height: int):
        """Receivers (H*W, 8) at a pinhole camera's primary hits, and the hit mask."""
        cam = np.ascontiguousarray(np.asarray(camera, np.float32).reshape(10))
        out = np.zeros((width * height, 8), np.float32)
        hit = np.zeros(width * height, np.uint8)
        check(load().cc_scene_primary_hits(self.handle, ptr(cam), int(width), int(height), ptr(out), ptr(hit)))
        return out, hit

    def close(self) -> None:
        if self._h:
            load().cc_scene_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def host_scene(meshes=None, tri9=None, counts=None) -> Scene:
    """A scene built on the host only (no device needed): hierarchies to
    inspect and ray cast, not to pass to ``visibility``."""
    if meshes is not None:
        tri9, counts = flatten_meshes(meshes)
    tri9 = np.ascontiguousarray(tri9, dtype=np.float32)
    counts = np.ascontiguousarray(counts, dtype=np.uint32)
    h = C.c_void_p()
    check(load().cc_scene_build(None, ptr(tri9), ptr(counts), len(counts), C.byref(h)))
    return Scene(None, h.value)


def instances_array(instances) -> np.ndarray:
    """cc_instance records from an INSTANCE_DTYPE array or (geometry, rotation
    3x3, scale, translation) tuples."""
    if isinstance(instances, np.ndarray) and instances.dtype == _lib.INSTANCE_DTYPE:
        return np.ascontiguousarray(instances)
    out = np.zeros(len(instances), _lib.INSTANCE_DTYPE)
    for i, (g, rot, scale, t) in enumerate(instances):
        out[i] = (g, np.asarray(rot, np.float32).reshape(9), scale, np.asarray(t, np.float32).reshape(3))
    return out


def _build_instanced(handle, geometries, instances, movable=None) -> int:
    tri9, counts = flatten_meshes(geometries)
    inst = instances_array(instances)
    mov = None if movable is None else np.ascontiguousarray(movable, np.uint32)
    h = C.c_void_p()
    check(load().cc_scene_build_instanced(handle, ptr(tri9), ptr(counts), len(counts), ptr(inst), len(inst), ptr(mov),
                                          0 if mov is None else len(mov), C.byref(h)))
    return h.value


def host_scene_instanced(geometries, instances, movable=None) -> Scene:
    """An instanced scene built on the host only (hierarchies to inspect and
    ray cast)."""
    return Scene(None, _build_instanced(None, geometries, instances, movable))


class MaskConeKernel:
    """Mask-cone visibility on one CUDA device (MaskConeKernel, lib.rs:65-120).

    Like the reference's kernel it is used from one thread at a time. The walk
    parameters the reference keeps in cells (``wide_extent``,
    ``light_cone_cap``, ``wide_cone_cap``; lib.rs:1211-1213; ``prefilter``,
    set_prefilter, lib.rs:1508; ``object_prefilter``, lib.rs:1595) are
    attributes.
    """

    def __init__(self, device: int = 0):
        lib = load()
        h = C.c_void_p()
        check(lib.cc_context_create(int(device), C.byref(h)))
        self._h = h
        self.device = device
        self.wide_extent = 8.0
        self.light_cone_cap = 4096
        self.wide_cone_cap = 512
        self.points_per_warp = 32
        self.prefilter = 0.0
        self.object_prefilter = True

    def set_split_chunk(self, cones: int) -> None:
        """Cones one chunk of the split path holds at most (its device scratch
        is 368 bytes a slot); results do not depend on it
        (cc_context_set_split_chunk)."""
        check(load().cc_context_set_split_chunk(self.handle, int(cones)))

    @classmethod
    def new(cls, device: int = 0) -> Optional["MaskConeKernel"]:
        """None without a CUDA device, as MaskConeKernel::new (lib.rs:1155-1175)."""
        try:
            return cls(device)
        except CCError as e:
            if e.code == _lib.CC_ERR_NO_DEVICE:
                return None
            raise

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise ValueError("kernel is closed")
        return self._h

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().cc_context_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the reference's calls ---------------------------------------------------
    def irradiance(self, receivers, light: RectLight, meshes, runs: int = 1):
        """Irradiance per unit radiance at each receiver and the best of `runs`
        kernel times in seconds; every receiver tests every mesh (lib.rs:1706-1715)."""
        return self.irradiance_with(receivers, light, meshes, Hierarchy.NONE, runs)

    def irradiance_with(self, receivers, light: RectLight, meshes, hierarchy, runs: int = 1):
        """`irradiance` culling through the hierarchy (lib.rs:1718-1730)."""
        rec = np.ascontiguousarray(np.asarray(receivers, dtype=np.float32).reshape(-1, 6))
        l9 = np.concatenate([_v3(light.corner), _v3(light.edge_u), _v3(light.edge_v)]).astype(np.float32)
        tri9, counts = flatten_meshes(meshes)
        out = np.zeros(rec.shape[0], dtype=np.float32)
        best = C.c_double(0.0)
        check(load().cc_irradiance(self.handle, ptr(rec), rec.shape[0], ptr(l9), int(bool(light.one_sided)),
                                   ptr(tri9), ptr(counts), len(counts), int(Hierarchy.of(hierarchy)), int(runs),
                                   ptr(out), C.byref(best)))
        return out, best.value

    def coverage(self, receivers, light: RectLight, meshes) -> np.ndarray:
        """Per-bin coverage (64 per receiver), every triangle tested (lib.rs:3289-3298)."""
        rec = np.ascontiguousarray(np.asarray(receivers, dtype=np.float32).reshape(-1, 6))
        l9 = np.concatenate([_v3(light.corner), _v3(light.edge_u), _v3(light.edge_v)]).astype(np.float32)
        tri9, counts = flatten_meshes(meshes)
        out = np.zeros((rec.shape[0], 64), dtype=np.float32)
        check(load().cc_coverage(self.handle, ptr(rec), rec.shape[0], ptr(l9), int(bool(light.one_sided)),
                                 ptr(tri9), ptr(counts), len(counts), ptr(out)))
        return out

    # -- resident scenes and the multi-light call -----------------------------------
    def scene(self, meshes) -> Scene:
        """Builds the hierarchies on the host and uploads the scene."""
        tri9, counts = flatten_meshes(meshes)
        return self.scene_from_tri9(tri9, counts)

    def scene_instanced(self, geometries, instances, movable=None) -> Scene:
        """An instanced scene: shared geometries (object space) placed by
        transforms (flatten_instanced, hierarchy.rs:464-522); `movable`
        objects keep a subtree of their own (Scene.move places them anew)."""
        return Scene(self, _build_instanced(self.handle, geometries, instances, movable))

    def stale_cones(self, scene: Scene, d_receivers: int, npoints: int, lights: np.ndarray, boxes: np.ndarray,
                    d_stale: int, stream: int = 0) -> int:
        """Marks (1 byte per cone, device) the cones the moved boxes may have
        changed; returns their count. lights and boxes are host arrays."""
        lig = np.ascontiguousarray(lights, np.float32).reshape(-1, 16)
        b = np.ascontiguousarray(boxes, np.float32).reshape(-1, 12)
        n = C.c_uint64()
        check(load().cc_stale_cones(self.handle, scene.handle, C.c_void_p(d_receivers), int(npoints), ptr(lig),
                                    lig.shape[0], ptr(b), b.shape[0], C.c_void_p(d_stale), C.byref(n),
                                    C.c_void_p(stream) if stream else None))
        return int(n.value)

    def visibility_update(self, scene: Scene, d_receivers: int, npoints: int, d_lights: int, nlights: int,
                          d_stale: int, outputs: dict, hierarchy=Hierarchy.TRIANGLES, stream: int = 0) -> int:
        """Recomputes the stale cones of device result arrays in place;
        returns the cones solved."""
        o = _lib.Outputs(*(outputs.get(k) for k in ("full", "any", "partial", "irradiance", "fraction", "work")))
        opt = self.options(hierarchy)
        n = C.c_uint64()
        check(load().cc_visibility_update(self.handle, scene.handle, C.c_void_p(d_receivers), int(npoints),
                                          C.c_void_p(d_lights), int(nlights), C.c_void_p(d_stale), C.byref(opt),
                                          C.byref(o), C.byref(n), C.c_void_p(stream) if stream else None))
        return int(n.value)

    def scene_from_tri9(self, tri9: np.ndarray, counts: np.ndarray) -> Scene:
        tri9 = np.ascontiguousarray(tri9, dtype=np.float32)
        counts = np.ascontiguousarray(counts, dtype=np.uint32)
        h = C.c_void_p()
        check(load().cc_scene_build(self.handle, ptr(tri9), ptr(counts), len(counts), C.byref(h)))
        return Scene(self, h.value)

    def scene_from_flat(self, tris12, ranges, blas, blas_items, nodes, items) -> Scene:
        """A scene from the reference's own flattened arrays (Flat + mesh_hierarchy)."""
        arrs = [np.ascontiguousarray(tris12, np.float32), np.ascontiguousarray(ranges, np.uint32),
                np.ascontiguousarray(blas), np.ascontiguousarray(blas_items, np.uint32),
                np.ascontiguousarray(nodes), np.ascontiguousarray(items, np.uint32)]
        f = _lib.FlatScene(ptr(arrs[0]), arrs[0].size // 12, ptr(arrs[1]), arrs[1].size // 4, ptr(arrs[2]),
                           len(arrs[2]), ptr(arrs[3]), arrs[3].size, ptr(arrs[4]), len(arrs[4]), ptr(arrs[5]),
                           arrs[5].size, None, 0)
        h = C.c_void_p()
        check(load().cc_scene_upload(self.handle, C.byref(f), C.byref(h)))
        return Scene(self, h.value)

    def options(self, hierarchy=Hierarchy.TRIANGLES, flags: int = 0, points_per_warp: Optional[int] = None):
        o = _lib.default_options()
        o.hierarchy = int(Hierarchy.of(hierarchy))
        o.wide_extent = float(self.wide_extent)
        o.light_cone_cap = int(self.light_cone_cap)
        o.wide_cone_cap = int(self.wide_cone_cap)
        o.points_per_warp = int(points_per_warp or self.points_per_warp)
        o.flags = int(flags) | (0 if self.object_prefilter else _lib.CC_NO_OBJECT_PREFILTER)
        o.prefilter = float(self.prefilter)
        return o

    def visibility(self, scene: Scene, receivers, lights, hierarchy=Hierarchy.TRIANGLES,
                   outputs: Sequence[str] = ("full", "any", "irradiance", "fraction"),
                   points_per_warp: Optional[int] = None, flags: int = 0) -> Visibility:
        """Every (light, point) cone through a resident scene; results [L, P]."""
        rec = receivers_gpu(receivers)
        lig = lights if isinstance(lights, np.ndarray) else lights_gpu(lights)
        lig = np.ascontiguousarray(lig, dtype=np.float32).reshape(-1, 16)
        P, L = rec.shape[0], lig.shape[0]
        res = Visibility()
        bufs = {}
        if "full" in outputs:
            bufs["full"] = np.zeros((L, P), np.uint64)
        if "any" in outputs:
            bufs["any"] = np.zeros((L, P), np.uint64)
        if "partial" in outputs:
            bufs["partial"] = np.zeros((L, P, 64), np.float32)
        if "irradiance" in outputs:
            bufs["irradiance"] = np.zeros((L, P), np.float32)
        if "fraction" in outputs:
            bufs["fraction"] = np.zeros((L, P), np.float32)
        if "work" in outputs:
            bufs["work"] = np.zeros((L, P, 4), np.uint32)
        o = _lib.Outputs(*(ptr(bufs.get(k)) for k in ("full", "any", "partial", "irradiance", "fraction", "work")))
        opt = self.options(hierarchy, flags, points_per_warp)
        check(load().cc_visibility(self.handle, scene.handle, ptr(rec), P, ptr(lig), L, C.byref(opt), C.byref(o),
                                   None))
        for k, v in bufs.items():
            setattr(res, k, v)
        return res

    def visibility_device(self, scene: Scene, d_receivers: int, npoints: int, d_lights: int, nlights: int,
                          outputs: dict, stream: int = 0, hierarchy=Hierarchy.TRIANGLES,
                          points_per_warp: Optional[int] = None, flags: int = 0) -> None:
        """The same with device pointers (ints), asynchronous on `stream`."""
        o = _lib.Outputs(*(outputs.get(k) for k in ("full", "any", "partial", "irradiance", "fraction", "work")))
        opt = self.options(hierarchy, flags | _lib.CC_DEVICE_POINTERS, points_per_warp)
        check(load().cc_visibility(self.handle, scene.handle, C.c_void_p(d_receivers), int(npoints),
                                   C.c_void_p(d_lights), int(nlights), C.byref(opt), C.byref(o),
                                   C.c_void_p(stream) if stream else None))

    def sky_visibility(self, scene: Scene, receivers, hierarchy=Hierarchy.TRIANGLES, sky_flags: int = 0,
                       outputs: Sequence[str] = (), points_per_warp: Optional[int] = None, flags: int = 0):
        """Sky cones (cc_sky_visibility): the irradiance per unit uniform sky
        radiance per receiver, and with `outputs` the six face cones' results
        [6, P] (face-major) in a Visibility."""
        rec = receivers_gpu(receivers)
        P = rec.shape[0]
        irr = np.zeros(P, np.float32)
        faces = Visibility()
        bufs = {}
        shapes = {"full": ((6, P), np.uint64), "any": ((6, P), np.uint64), "partial": ((6, P, 64), np.float32),
                  "irradiance": ((6, P), np.float32), "fraction": ((6, P), np.float32), "work": ((6, P, 4), np.uint32)}
        for k in outputs:
            shape, dt = shapes[k]
            bufs[k] = np.zeros(shape, dt)
        o = _lib.Outputs(*(ptr(bufs.get(k)) for k in ("full", "any", "partial", "irradiance", "fraction", "work")))
        opt = self.options(hierarchy, flags, points_per_warp)
        check(load().cc_sky_visibility(self.handle, scene.handle, ptr(rec), P, C.byref(opt), int(sky_flags), ptr(irr),
                                       C.byref(o) if bufs else None, None))
        for k, v in bufs.items():
            setattr(faces, k, v)
        return irr, faces

    def sky_visibility_device(self, scene: Scene, d_receivers: int, npoints: int, d_irradiance: int,
                              faces: Optional[dict] = None, stream: int = 0, hierarchy=Hierarchy.TRIANGLES,
                              sky_flags: int = 0, points_per_warp: Optional[int] = None, flags: int = 0) -> None:
        """The same with device pointers (ints), asynchronous on `stream`."""
        o = None
        if faces:
            o = _lib.Outputs(*(faces.get(k) for k in ("full", "any", "partial", "irradiance", "fraction", "work")))
        opt = self.options(hierarchy, flags | _lib.CC_DEVICE_POINTERS, points_per_warp)
        check(load().cc_sky_visibility(self.handle, scene.handle, C.c_void_p(d_receivers), int(npoints), C.byref(opt),
                                       int(sky_flags), C.c_void_p(d_irradiance), C.byref(o) if o else None,
                                       C.c_void_p(stream) if stream else None))

    def visibility_static(self, scene: Scene, d_receivers: int, npoints: int, d_lights: int, nlights: int,
                          outputs: dict, stream: int = 0, hierarchy=Hierarchy.TRIANGLES,
                          points_per_warp: Optional[int] = None, flags: int = 0) -> None:
        """visibility_device through cc_visibility_static: no allocation, at
        most CC_STATIC_MAX_CONES cones, one call in flight per device."""
        o = _lib.Outputs(*(outputs.get(k) for k in ("full", "any", "partial", "irradiance", "fraction", "work")))
        opt = self.options(hierarchy, flags | _lib.CC_DEVICE_POINTERS, points_per_warp)
        check(load().cc_visibility_static(scene.handle, C.c_void_p(d_receivers), int(npoints), C.c_void_p(d_lights),
                                          int(nlights), C.byref(opt), C.byref(o),
                                          C.c_void_p(stream) if stream else None))


class Batch:
    """Many visibility jobs solved by one persistent launch (cc_batch_*).

    Jobs take device pointers (ints) for their receivers, lights and outputs,
    which must stay valid while the batch is submitted. Each job's results
    equal a visibility_device call for that job alone.
    """

    def __init__(self, kernel: MaskConeKernel):
        h = C.c_void_p()
        check(load().cc_batch_create(kernel.handle, C.byref(h)))
        self._h = h
        self.kernel = kernel

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise ValueError("batch is closed")
        return self._h

    def add(self, scene: Scene, d_receivers: int, npoints: int, d_lights: int, nlights: int, outputs: dict,
            hierarchy=Hierarchy.TRIANGLES, prefilter: Optional[float] = None) -> int:
        """A job (cc_batch_add); prefilter (bins; None: the kernel's setting)
        makes it a prefiltering job."""
        o = _lib.Outputs(*(outputs.get(k) for k in ("full", "any", "partial", "irradiance", "fraction", "work")))
        opt = self.kernel.options(hierarchy)
        if prefilter is not None:
            opt.prefilter = float(prefilter)
        job = C.c_uint32()
        check(load().cc_batch_add(self.handle, scene.handle, C.c_void_p(d_receivers), int(npoints),
                                  C.c_void_p(d_lights), int(nlights), C.byref(opt), C.byref(o), C.byref(job)))
        return int(job.value)

    def add_update(self, scene: Scene, d_receivers: int, npoints: int, d_lights: int, nlights: int, d_stale: int,
                   outputs: dict, hierarchy=Hierarchy.TRIANGLES) -> int:
        """An update job (cc_batch_add_update): each submission recomputes the
        cones whose byte in the device array `d_stale` (light-major) is set,
        in place in the device outputs (full, any, irradiance, fraction)."""
        o = _lib.Outputs(*(outputs.get(k) for k in ("full", "any", "partial", "irradiance", "fraction", "work")))
        opt = self.kernel.options(hierarchy)
        job = C.c_uint32()
        check(load().cc_batch_add_update(self.handle, scene.handle, C.c_void_p(d_receivers), int(npoints),
                                         C.c_void_p(d_lights), int(nlights), C.c_void_p(d_stale), C.byref(opt),
                                         C.byref(o), C.byref(job)))
        return int(job.value)

    @staticmethod
    def options(points_per_warp: int = 32, blocks_per_sm: int = 8, flags: int = _lib.CC_BATCH_GRAPH):
        return _lib.BatchOptions(int(points_per_warp), int(blocks_per_sm), int(flags))

    def submit(self, options=None, stream: int = 0) -> None:
        opt = options if options is not None else self.options()
        check(load().cc_batch_submit(self.handle, C.byref(opt), C.c_void_p(stream) if stream else None))

    def wait(self, timeout_ms: int = 600_000) -> None:
        check(load().cc_batch_wait(self.handle, int(timeout_ms)))

    def tune(self, reps: int = 2, flags: int = _lib.CC_BATCH_GRAPH):
        """The autotuner: (best options, each candidate's milliseconds)."""
        base = self.options(flags=flags)
        best = _lib.BatchOptions()
        ms = np.zeros(64, np.float32)
        n = load().cc_batch_tune(self.handle, C.byref(base), int(reps), C.byref(best), ptr(ms), 64)
        if n < 0:
            check(-n)
        return best, ms[:n]

    def sizes(self) -> dict:
        out = np.zeros(4, np.uint64)
        check(load().cc_batch_sizes(self.handle, ptr(out)))
        return {"jobs": int(out[0]), "points": int(out[1]), "cones": int(out[2]), "device_bytes": int(out[3])}

    def clear(self) -> None:
        check(load().cc_batch_clear(self.handle))

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().cc_batch_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The served form (cc_server_*): a native request loop with continuous
    batching, admission against a device-memory budget (reserved when the
    server is made), earliest deadline first (deadline_ns_per_cone per cone
    after submission; 0: arrival order), and a resident lighting cache.
    Requests take host arrays, which the server's thread reads and writes
    until the request completes (pinned memory lets the copies overlap with
    other launches; a copy to pageable memory holds the server's thread until
    its launch is done)."""

    def __init__(self, kernel: MaskConeKernel, hbm_budget: int = 8 << 30, max_inflight: int = 4,
                 max_queue: int = 256, max_launch_cones: int = 2 << 20, points_per_warp: int = 32,
                 blocks_per_sm: int = 8, deadline_ns_per_cone: int = 12):
        opt = _lib.ServerOptions(int(hbm_budget), int(max_inflight), int(max_queue), int(max_launch_cones),
                                 int(points_per_warp), int(blocks_per_sm), int(deadline_ns_per_cone))
        h = C.c_void_p()
        check(load().cc_server_create(kernel.handle, C.byref(opt), C.byref(h)))
        self._h = h
        self.kernel = kernel
        self._live = {}  # ticket -> the arrays the request reads and writes

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise ValueError("server is closed")
        return self._h

    def add_scene(self, scene: Scene) -> int:
        i = C.c_uint32()
        check(load().cc_server_add_scene(self.handle, scene.handle, C.byref(i)))
        return int(i.value)

    def submit(self, scene_id: int, receivers: np.ndarray, lights: np.ndarray, outputs: dict,
               hierarchy=Hierarchy.TRIANGLES, cache_key: int = 0, prefilter: float = 0.0) -> int:
        """Queues a request; outputs maps full/any (uint64 [L, P]) and
        irradiance/fraction (float32 [L, P]) to host arrays. Raises CCError
        (CC_ERR_BUSY) when the queue is full."""
        rec = np.ascontiguousarray(receivers, np.float32)
        lig = np.ascontiguousarray(lights, np.float32).reshape(-1, 16)
        for k, v in outputs.items():
            if not v.flags["C_CONTIGUOUS"] or v.size < rec.shape[0] * lig.shape[0]:
                raise ValueError(f"output {k} must be C-contiguous with a value per cone")
        req = _lib.Request(int(scene_id), ptr(rec), rec.shape[0], ptr(lig), lig.shape[0],
                           int(Hierarchy.of(hierarchy)), int(cache_key),
                           *(ptr(outputs.get(k)) for k in ("full", "any", "irradiance", "fraction")),
                           float(prefilter))
        t = C.c_uint64()
        check(load().cc_server_submit(self.handle, C.byref(req), C.byref(t)))
        self._live[int(t.value)] = (rec, lig, outputs)
        return int(t.value)

    def wait(self, ticket: int, timeout_ms: int = 600_000) -> dict:
        st = _lib.RequestStats()
        try:
            check(load().cc_server_wait(self.handle, int(ticket), int(timeout_ms), C.byref(st)))
        except CCError as e:
            if e.code != _lib.CC_ERR_TIMEOUT:
                self._live.pop(int(ticket), None)
            raise
        self._live.pop(int(ticket), None)
        return {"queued_ms": st.queued_ms, "total_ms": st.total_ms, "launch_requests": st.launch_requests,
                "cached_lights": st.cached_lights}

    def stats(self) -> dict:
        out = np.zeros(8, np.uint64)
        check(load().cc_server_stats(self.handle, ptr(out)))
        keys = ("completed", "refused", "launches", "cached_lights", "traced_lights", "bytes_in_use", "peak_bytes",
                "cache_entries")
        return {k: int(v) for k, v in zip(keys, out)}

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().cc_server_destroy(self._h)
            self._h = C.c_void_p(None)
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kernel_times(kernel: MaskConeKernel, max_calls: int = 256) -> np.ndarray:
    """(calls, 2) milliseconds of the packet and solo passes of the
    visibility calls since the last query (waits for them)."""
    out = np.zeros((max_calls, 2), np.float32)
    n = load().cc_context_kernel_times(kernel.handle, ptr(out), int(max_calls))
    if n < 0:
        check(-n)
    return out[:n]


# ---- the lighting cache's bake ---------------------------------------------------

PAGE_TEXELS = 81  # 8 x 8 texels stored 9 x 9 (vcache.rs:32-35)
#: Texel flags (the w of a texel record's point): outside the chart's grid,
#: inside without a surface, a surface to bake.
TEXEL_OUTSIDE, TEXEL_EMPTY, TEXEL_SURFACE = 0.0, 1.0, 2.0


@dataclass
class PageRequest:
    """A page a view wants (vcache.rs: a request with its priority): `key` of
    3 u32, `priority` (lower first), `inside` texels per axis (0..9) and
    `texels`, 81 x 8 floats (point.xyz, flag, normal.xyz, own triangle + 1
    as uint32 bits or 0), row-major 9 x 9, needed only when the page is not
    resident."""

    key: Sequence[int]
    priority: int
    inside: Sequence[int] = (8, 8)
    texels: Optional[np.ndarray] = None


def cache_options(pages: int = 1 << 16, bake_budget: int = 1 << 20, frame_target_ms: float = 0.0,
                  frame_budget_ms: float = 0.0, floor_overrun: float = 0.25, light_ratio: bool = True):
    return _lib.CacheOptions(int(pages), int(bake_budget), float(frame_target_ms), float(frame_budget_ms),
                             float(floor_overrun), 1 if light_ratio else 0)


class PreparedRequests:
    """Page requests converted once for the C ABI, for a view that asks for
    the same pages frame after frame."""

    def __init__(self, reqs: Sequence[PageRequest]):
        self.arr, self.keep = _requests(reqs)
        self.n = len(reqs)


def prepare_requests(reqs: Sequence[PageRequest]) -> PreparedRequests:
    return PreparedRequests(reqs)


def _requests(reqs):
    if isinstance(reqs, PreparedRequests):
        return reqs.arr, reqs.keep
    arr = (_lib.PageRequest * max(len(reqs), 1))()
    keep = []
    for i, r in enumerate(reqs):
        arr[i].key[:] = [int(x) for x in r.key]
        arr[i].priority = int(r.priority)
        arr[i].inside[:] = [int(x) for x in r.inside]
        if r.texels is not None:
            t = np.ascontiguousarray(r.texels, dtype=np.float32).reshape(PAGE_TEXELS, 8)
            keep.append(t)
            arr[i].texels = t.ctypes.data
        else:
            arr[i].texels = None
    return arr, keep


def _count(reqs) -> int:
    return reqs.n if isinstance(reqs, PreparedRequests) else len(reqs)


def _stats(s: _lib.CacheStats) -> dict:
    return {k: getattr(s, k) for k, _ in _lib.CacheStats._fields_}


def _frame_info(period_ms: float, render_ms: float, gpu_waited: bool):
    return _lib.CacheFrameInfo(float(period_ms), float(render_ms), 1 if gpu_waited else 0)


def _jobs(fn, handle, max_pages: int = 1 << 20):
    n = fn(handle, None, 0, None, 0)
    if n < 0:
        check(int(-n))
    jobs = np.zeros((max(n, 1), 2), np.uint32)
    slots = np.zeros(max_pages, np.uint32)
    fn(handle, ptr(jobs), int(n), ptr(slots), int(max_pages))
    return jobs[:n], slots


class Planner:
    """The lighting cache's page manager alone, on the host (cc_planner_*):
    each frame plans the requested pages within the bake budget, adapts the
    budget to the frame time from the bake's measured GPU time, and lists the
    bake jobs [bake-list index, texel | light << 8]."""

    def __init__(self, nlights: int = 1, **options):
        h = C.c_void_p()
        opt = cache_options(**options)
        check(load().cc_planner_create(C.byref(opt), int(nlights), C.byref(h)))
        self._h = h
        self.nlights = nlights

    def frame(self, requests: Sequence[PageRequest], period_ms: float = 0.0, render_ms: float = 0.0,
              gpu_waited: bool = False, bake_ms: float = -1.0) -> dict:
        arr, _keep = _requests(requests)
        st = _lib.CacheStats()
        info = _frame_info(period_ms, render_ms, gpu_waited)
        check(load().cc_planner_frame(self._h, arr, _count(requests), C.byref(info), float(bake_ms), C.byref(st)))
        return _stats(st)

    def jobs(self):
        """(jobs (n, 2) u32, slot per planned page) of the last frame."""
        jobs, slots = _jobs(load().cc_planner_jobs, self._h)
        return jobs, slots[: (int(jobs[:, 0].max()) + 1) if len(jobs) else 0]

    def slot(self, key) -> int:
        k = np.asarray(key, np.uint32)
        return int(load().cc_planner_slot(self._h, ptr(k)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().cc_planner_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LightingCache:
    """The lighting cache's direct-light bake on the device (cc_cache_*): a
    pool of pages, one channel per light, baked frame by frame from the
    view's page requests within the bake budget."""

    def __init__(self, kernel: MaskConeKernel, scene: Scene, lights, **options):
        self.kernel, self.scene = kernel, scene
        self.lights = np.ascontiguousarray(lights_gpu(lights) if not isinstance(lights, np.ndarray) else lights,
                                           dtype=np.float32).reshape(-1, 16)
        h = C.c_void_p()
        opt = cache_options(**options)
        check(load().cc_cache_create(kernel.handle, scene.handle, ptr(self.lights), self.lights.shape[0],
                                     C.byref(opt), C.byref(h)))
        self._h = h

    @property
    def nlights(self) -> int:
        return self.lights.shape[0]

    def frame(self, requests: Sequence[PageRequest], period_ms: float = 0.0, render_ms: float = 0.0,
              gpu_waited: bool = False) -> dict:
        arr, _keep = _requests(requests)
        st = _lib.CacheStats()
        info = _frame_info(period_ms, render_ms, gpu_waited)
        check(load().cc_cache_frame(self._h, arr, _count(requests), C.byref(info), C.byref(st)))
        return _stats(st)

    def read(self, key) -> np.ndarray:
        """A resident page's (81, nlights) pool values."""
        k = np.asarray(key, np.uint32)
        out = np.zeros((PAGE_TEXELS, self.nlights), np.float32)
        check(load().cc_cache_read(self._h, ptr(k), ptr(out)))
        return out

    def jobs(self):
        jobs, slots = _jobs(load().cc_cache_jobs, self._h)
        return jobs, slots[: (int(jobs[:, 0].max()) + 1) if len(jobs) else 0]

    def pool(self) -> tuple[int, int]:
        p, ch = C.c_void_p(), C.c_uint32()
        check(load().cc_cache_pool(self._h, C.byref(p), C.byref(ch)))
        return int(p.value or 0), int(ch.value)

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().cc_cache_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
