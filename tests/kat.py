"""Fixtures of the reference's own known-answer tests for the mask-cone path.

Each builder reproduces a scene from the reference's tests (cited), in the
reference's frame (+Z up), as plain numpy arrays for both the oracle and the
CUDA library.
"""
from __future__ import annotations

import math

import numpy as np

from continuum_b200.kernel import Light, RectLight, light_gpu
from continuum_b200.scenes import Pcg32, box_mesh, sphere_mesh

# The 0.2 x 0.2 ceiling light at height 1 of the reference's cone tests
# (cone3.rs:503-513, gpu.rs:305-310, room3d gate1 lib.rs:83-87).
CEILING = RectLight(corner=(0.4, 0.4, 1.0), edge_u=(0.2, 0.0, 0.0), edge_v=(0.0, 0.2, 0.0), one_sided=False)


def light9(rect: RectLight) -> np.ndarray:
    return np.concatenate([np.asarray(rect.corner, np.float32), np.asarray(rect.edge_u, np.float32),
                           np.asarray(rect.edge_v, np.float32)]).astype(np.float32)


def receivers(points, normals) -> np.ndarray:
    p = np.asarray(points, np.float32).reshape(-1, 3)
    n = np.broadcast_to(np.asarray(normals, np.float32), p.shape)
    out = np.zeros((p.shape[0], 8), np.float32)
    out[:, 0:3] = p
    out[:, 4:7] = n
    return out


def four_boxes():
    """cones_match_the_cpu (crates/continuum-gltf/tests/gpu.rs:294-337)."""
    return [
        box_mesh((0.30, 0.10, 0.55), (0.70, 0.35, 0.58)),
        box_mesh((0.62, 0.40, 0.30), (0.85, 0.60, 0.33)),
        box_mesh((0.15, 0.45, 0.20), (0.25, 0.55, 0.30)),
        box_mesh((0.40, 0.65, 0.45), (0.48, 0.90, 0.62)),
    ]


def grid_floor(size: int) -> np.ndarray:
    """Receivers ((i+0.5)/size, (j+0.5)/size, 0), normal +Z (gpu.rs:312-322)."""
    k = np.arange(size * size)
    i, j = k % size, k // size
    pts = np.stack([(i + 0.5) / size, (j + 0.5) / size, np.zeros_like(i, dtype=np.float64)], axis=1)
    return receivers(pts.astype(np.float32), (0.0, 0.0, 1.0))


def gate1_room():
    """The M2 gate 1 room (experiments/room3d/src/lib.rs:56-89): four fences of
    thin slats, a table top, a floating cube."""
    meshes = []

    def slats(y0, y1, z, shift):
        for i in range(8):
            x = np.float32(0.30) + np.float32(i) * np.float32(0.04) + np.float32(shift)
            meshes.append(box_mesh((x, y0, z), (x + np.float32(0.02), y1, z + np.float32(0.01))))

    slats(0.10, 0.35, 0.55, 0.0)
    slats(0.10, 0.35, 0.62, 0.0)
    slats(0.65, 0.90, 0.55, 0.0)
    slats(0.65, 0.90, 0.62, 0.02)
    meshes.append(box_mesh((0.62, 0.40, 0.30), (0.85, 0.60, 0.33)))
    meshes.append(box_mesh((0.15, 0.45, 0.20), (0.25, 0.55, 0.30)))
    return meshes


def floor_points(size: int) -> np.ndarray:
    """floor_point (room3d lib.rs:44-52): row-major, y up the image."""
    k = np.arange(size * size)
    i, j = k % size, k // size
    pts = np.stack([(i + 0.5) / size, 1.0 - (j + 0.5) / size, np.zeros(size * size)], axis=1)
    return receivers(pts.astype(np.float32), (0.0, 0.0, 1.0))


def with_rubble(count: int = 3000):
    """Gate 1 plus small boxes scattered under the fences (room3d lib.rs:98-119), PCG32(42, 7)."""
    meshes = gate1_room()
    rng = Pcg32(42, 7)
    for _ in range(count):
        p = np.array([0.05 + 0.9 * rng.next_f32(), 0.05 + 0.9 * rng.next_f32(), 0.35 + 0.15 * rng.next_f32()],
                     np.float32)
        s = np.array([0.01 + 0.01 * rng.next_f32(), 0.01 + 0.01 * rng.next_f32(), 0.01 + 0.01 * rng.next_f32()],
                     np.float32)
        meshes.append(box_mesh(p, p + s))
    return meshes


def with_sphere(segments=200, rings=100):
    """Gate 1 plus a finely tessellated sphere (room3d lib.rs:91-96)."""
    return gate1_room() + [sphere_mesh((0.3, 0.72, 0.45), 0.08, segments, rings)]


def wall():
    """A wall of two 20 m triangles in the plane x = 0 facing +x (gpu.rs:339-345)."""
    c = [np.array([0.0, y, z], np.float32) for (y, z) in [(-10.0, -10.0), (10.0, -10.0), (10.0, 10.0), (-10.0, 10.0)]]
    return [np.asarray([[c[0], c[1], c[2]], [c[0], c[2], c[3]]], np.float32)]


def distant_light(center, toward, distance, solid_angle) -> RectLight:
    """Light::distant's rectangle (crates/continuum-gpu/src/lib.rs:672-703), in f64 then f32."""
    toward = np.asarray(toward, np.float64)
    toward = toward / np.linalg.norm(toward)
    size = distance * math.sqrt(max(solid_angle, 1e-12))
    w = -toward
    z = np.array([0.0, 0.0, 1.0])
    side = np.cross(z, w) if np.linalg.norm(np.cross(w, z)) > 1e-6 else np.array([1.0, 0.0, 0.0])
    a = side / np.linalg.norm(side) * size
    b = np.cross(w, a)
    b = b / np.linalg.norm(b) * size
    middle = np.asarray(center, np.float64) + toward * distance
    corner = middle - (a + b) * 0.5
    return RectLight(tuple(corner.astype(np.float32)), tuple(a.astype(np.float32)), tuple(b.astype(np.float32)),
                     one_sided=True)


def sun_behind_the_wall() -> RectLight:
    """gpu.rs:347-355: Light::sun(ZERO, (-0.6, -0.3, 0.75), 900, ...)."""
    size = 2.0 * math.tan(math.radians(0.25))
    return distant_light((0.0, 0.0, 0.0), (-0.6, -0.3, 0.75), 900.0, size * size)


def wall_receivers() -> np.ndarray:
    """gpu.rs:365-374: 20 x 20 receivers with normals between up and toward the wall."""
    pts, nrm = [], []
    for k in range(400):
        i, j = k % 20, k // 20
        pts.append([0.02 + 0.03 * i, -1.0 + 0.1 * j, 0.5])
        n = np.array([-0.05 * i, 0.0, 1.0])
        nrm.append(n / np.linalg.norm(n))
    out = np.zeros((400, 8), np.float32)
    out[:, 0:3] = np.asarray(pts, np.float32)
    out[:, 4:7] = np.asarray(nrm, np.float32)
    return out


def lights16(*rects) -> np.ndarray:
    return np.stack([light_gpu(Light.rect(r)) for r in rects]).astype(np.float32)


def ray_triangle(origin, d, tris):
    """Distances along d to each triangle (Moller-Trumbore), inf where missed; vectorised over tris."""
    v0, v1, v2 = tris[:, 0].astype(np.float64), tris[:, 1].astype(np.float64), tris[:, 2].astype(np.float64)
    e1, e2 = v1 - v0, v2 - v0
    p = np.cross(d, e2)
    det = np.einsum("ij,ij->i", e1, p)
    ok = np.abs(det) >= 1e-12
    inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
    s = origin - v0
    u = np.einsum("ij,ij->i", s, p) * inv
    q = np.cross(s, e1)
    v = (q @ d) * inv
    t = np.einsum("ij,ij->i", e2, q) * inv
    hit = ok & (u >= 0) & (u <= 1) & (v >= 0) & (u + v <= 1) & (t > 0)
    return np.where(hit, t, np.inf)


def sampled_visible(p, meshes, n: int) -> float:
    """Stratified area sampling of the ceiling light, cosine at both ends (cone3.rs:516-537)."""
    p = np.asarray(p, np.float64)
    g = (np.arange(n) + 0.5) / n
    qi, qj = np.meshgrid(0.4 + 0.2 * g, 0.4 + 0.2 * g, indexing="ij")
    d = np.stack([qi.ravel() - p[0], qj.ravel() - p[1], np.full(n * n, 1.0 - p[2])], axis=1)  # (S, 3)
    blocked = np.zeros(n * n, bool)
    for m in meshes:
        for tri in np.asarray(m, np.float64):
            v0, v1, v2 = tri
            e1, e2 = v1 - v0, v2 - v0
            pv = np.cross(d, e2)
            det = pv @ e1
            ok = np.abs(det) >= 1e-12
            inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
            s = p - v0
            u = (pv @ s) * inv
            q = np.cross(s, e1)
            v = (d @ q) * inv
            t = (e2 @ q) * inv
            blocked |= ok & (u >= 0) & (u <= 1) & (v >= 0) & (u + v <= 1) & (t > 0) & (t < 1.0)
    r2 = np.einsum("ij,ij->i", d, d)
    cos = d[:, 2] / np.sqrt(r2)
    return float(np.sum(np.where(blocked, 0.0, cos * cos / r2)) * (0.04 / (n * n)))
