"""Seeded synthetic workloads for the visibility path.

Every generator is deterministic: PCG32 (O'Neill's public generator, which the
reference uses for its experiments, experiments/flatland/src/rng.rs:1-30)
drives all random choices. Geometry uses +Y up; the cone math is frame-free.

* ``box_field``: a 40 x 40 m ground quad and 64 axis-aligned boxes (edges
  U[0.2, 1] m, centres U[-8, 8] in x and z, resting on the ground), one 1 x 1 m
  one-sided rect light facing down at y = 4 m, and a 256 x 256 grid of
  receivers on the ground over [-10, 10]^2.
* ``icosphere_field``: displaced icospheres (subdivision 5, 20,480 triangles
  each) with radii U[0.5, 3] m and centres U[-50, 50]^2 resting on a ground
  quad, four lights (rects 2 x 1 and 4 x 4 m, disks of radius 0.5 and 1.5 m) at
  heights U[8, 20] m tilted up to 30 degrees from straight down, and the
  primary hits of a 1280 x 720 camera with a 60-degree vertical field of view.
  A disk light is a sphere light of the same radius (a sphere is seen as a
  disk from every point) with a spot along the disk's normal whose cut-off is
  90 degrees, so it emits on one side only.
* ``box_mesh`` / ``sphere_mesh``: the reference's fixture meshes
  (crates/continuum/src/cone3.rs:419-496), wound counter-clockwise seen from
  outside.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from functools import lru_cache
from typing import Optional

import numpy as np

from .kernel import Light, RectLight, SphereLight, Spot, light_gpu

MASK64 = (1 << 64) - 1


class Pcg32:
    """PCG32 (XSH RR), seeded as the reference seeds it (seed, stream)."""

    MULT = 6364136223846793005

    def __init__(self, seed: int, stream: int):
        self.state = 0
        self.inc = ((stream << 1) | 1) & MASK64
        self.next_u32()
        self.state = (self.state + seed) & MASK64
        self.next_u32()

    def next_u32(self) -> int:
        old = self.state
        self.state = (old * self.MULT + self.inc) & MASK64
        xorshifted = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xorshifted >> rot) | (xorshifted << ((-rot) & 31))) & 0xFFFFFFFF

    def next_f32(self) -> float:
        """Uniform in [0, 1) with 24 bits."""
        return float(np.float32((self.next_u32() >> 8) * (1.0 / 16777216.0)))

    def uniform(self, lo: float, hi: float) -> float:
        return lo + (hi - lo) * self.next_f32()


def box_mesh(lo, hi) -> np.ndarray:
    """An axis-aligned box as 12 outward-facing triangles (12, 3, 3)."""
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)

    def c(x, y, z):
        return np.array([hi[0] if x else lo[0], hi[1] if y else lo[1], hi[2] if z else lo[2]], np.float32)

    F, T = False, True
    quads = [
        [c(F, F, F), c(F, T, F), c(T, T, F), c(T, F, F)],  # -z
        [c(F, F, T), c(T, F, T), c(T, T, T), c(F, T, T)],  # +z
        [c(F, F, F), c(T, F, F), c(T, F, T), c(F, F, T)],  # -y
        [c(F, T, F), c(F, T, T), c(T, T, T), c(T, T, F)],  # +y
        [c(F, F, F), c(F, F, T), c(F, T, T), c(F, T, F)],  # -x
        [c(T, F, F), c(T, T, F), c(T, T, T), c(T, F, T)],  # +x
    ]
    tris = []
    for q in quads:
        tris.append([q[0], q[1], q[2]])
        tris.append([q[0], q[2], q[3]])
    return np.asarray(tris, np.float32)


def sphere_mesh(center, radius: float, segments: int, rings: int) -> np.ndarray:
    """A UV sphere with +Z poles as outward-facing triangles."""
    center = np.asarray(center, np.float32)

    def at(s, r):
        theta = np.float32(2 * math.pi) * np.float32(s) / np.float32(segments)
        phi = np.float32(math.pi) * np.float32(r) / np.float32(rings)
        return center + np.array([math.sin(phi) * math.cos(theta), math.sin(phi) * math.sin(theta), math.cos(phi)],
                                 np.float32) * np.float32(radius)

    tris = []
    for r in range(rings):
        for s in range(segments):
            a, b, cc, d = at(s, r), at(s + 1, r), at(s + 1, r + 1), at(s, r + 1)
            if r > 0:
                tris.append([a, d, b])
            if r + 1 < rings:
                tris.append([b, d, cc])
    return np.asarray(tris, np.float32)


def ground_quad(half: float, y: float = 0.0) -> np.ndarray:
    """Two triangles on y = `y` spanning [-half, half]^2, normal +y."""
    h = np.float32(half)
    a = [-h, y, -h]
    b = [-h, y, h]
    c = [h, y, h]
    d = [h, y, -h]
    return np.asarray([[a, b, c], [a, c, d]], np.float32)


@lru_cache(maxsize=None)
def unit_icosphere(subdivisions: int) -> np.ndarray:
    """Unit icosphere (20 * 4^n triangles, outward CCW) as (T, 3, 3) float64."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache = {}

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                m = verts[i] + verts[j]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.asarray(verts)
    F = np.asarray(faces)
    tris = V[F]
    # Outward winding: flip any face whose normal points inward.
    n = np.cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0])
    inward = np.einsum("ij,ij->i", n, tris.sum(axis=1)) < 0
    tris[inward] = tris[inward][:, ::-1]
    return tris


def _hash3(ix, iy, iz, seed: int) -> np.ndarray:
    """Lattice values in [-1, 1] from integer coordinates (a 32-bit mix)."""
    h = (ix.astype(np.int64) * 73856093) ^ (iy.astype(np.int64) * 19349663) ^ (iz.astype(np.int64) * 83492791)
    h = (h ^ (seed * 2654435761)) & 0xFFFFFFFF
    h = ((h ^ (h >> 16)) * 0x7FEB352D) & 0xFFFFFFFF
    h = ((h ^ (h >> 15)) * 0x846CA68B) & 0xFFFFFFFF
    h = h ^ (h >> 16)
    return (h.astype(np.float64) / 4294967295.0) * 2.0 - 1.0


def value_noise(p: np.ndarray, seed: int, octaves: int = 3) -> np.ndarray:
    """Seeded 3-octave value noise in about [-1, 1] at points p (N, 3)."""
    total = np.zeros(p.shape[0])
    amp, norm, freq = 1.0, 0.0, 1.0
    for o in range(octaves):
        q = p * freq
        i = np.floor(q).astype(np.int64)
        f = q - i
        f = f * f * (3 - 2 * f)
        acc = 0.0
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    w = (f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1]) * \
                        (f[:, 2] if dz else 1 - f[:, 2])
                    acc = acc + w * _hash3(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed + 1013 * o)
        total += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def displaced_icosphere(center, radius: float, seed: int, subdivisions: int = 5, amplitude: float = 0.15,
                        frequency: float = 2.0) -> np.ndarray:
    """An icosphere with vertices moved radially by seeded value noise of
    amplitude `amplitude` * radius."""
    unit = unit_icosphere(subdivisions)
    flat = unit.reshape(-1, 3)
    # Shared vertices displace alike: noise is a function of the unit position.
    scale = radius * (1.0 + amplitude * value_noise(flat * frequency, seed))
    pts = flat * scale[:, None] + np.asarray(center, np.float64)
    return pts.reshape(-1, 3, 3).astype(np.float32)


@dataclass
class Workload:
    """Meshes, lights (16-float records) and receivers (8 floats each)."""

    name: str
    meshes: list
    lights: np.ndarray
    receivers: Optional[np.ndarray] = None
    light_objects: Optional[list] = None
    camera: Optional[np.ndarray] = None
    size: Optional[tuple] = None

    def tri9(self):
        from .kernel import flatten_meshes
        return flatten_meshes(self.meshes)

    @property
    def ntris(self) -> int:
        return int(sum(len(m) for m in self.meshes))


def box_field(seed: int = 1, grid: int = 256) -> Workload:
    """The small plain workload: ground, 64 boxes, one rect light, grid receivers."""
    rng = Pcg32(seed, 11)
    meshes = [ground_quad(20.0)]
    for _ in range(64):
        e = [rng.uniform(0.2, 1.0) for _ in range(3)]
        cx, cz = rng.uniform(-8.0, 8.0), rng.uniform(-8.0, 8.0)
        meshes.append(box_mesh([cx - e[0] / 2, 0.0, cz - e[2] / 2], [cx + e[0] / 2, e[1], cz + e[2] / 2]))
    light = RectLight(corner=(-0.5, 4.0, -0.5), edge_u=(1.0, 0.0, 0.0), edge_v=(0.0, 0.0, 1.0), one_sided=True)
    lin = -10.0 + 20.0 * (np.arange(grid, dtype=np.float64) + 0.5) / grid
    zz, xx = np.meshgrid(lin, lin, indexing="ij")
    rec = np.zeros((grid * grid, 8), np.float32)
    rec[:, 0] = xx.reshape(-1)
    rec[:, 2] = zz.reshape(-1)
    rec[:, 5] = 1.0
    return Workload("box_field", meshes, light_gpu(Light.rect(light))[None, :], rec, [Light.rect(light)])


def _tilted_frame(rng: Pcg32, max_tilt_deg: float):
    """A unit normal within max_tilt of straight down (-y), and two edges' directions."""
    tilt = math.radians(max_tilt_deg) * rng.next_f32()
    az = 2 * math.pi * rng.next_f32()
    n = np.array([math.sin(tilt) * math.cos(az), -math.cos(tilt), math.sin(tilt) * math.sin(az)])
    helper = np.array([1.0, 0.0, 0.0]) if abs(n[0]) < 0.9 else np.array([0.0, 0.0, 1.0])
    u = np.cross(helper, n)
    u /= np.linalg.norm(u)
    v = np.cross(n, u)
    return n, u, v


def icosphere_field_lights(rng: Pcg32, spread: float = 40.0):
    lights = []
    specs = [("rect", 2.0, 1.0), ("rect", 4.0, 4.0), ("disk", 0.5, None), ("disk", 1.5, None)]
    for kind, a, b in specs:
        h = rng.uniform(8.0, 20.0)
        x, z = rng.uniform(-spread, spread), rng.uniform(-spread, spread)
        n, u, v = _tilted_frame(rng, 30.0)
        centre = np.array([x, h, z])
        if kind == "rect":
            # edge_u x edge_v along n (the light emits toward its normal).
            eu, ev = u * a, v * b
            if np.dot(np.cross(eu, ev), n) < 0:
                ev = -ev
            corner = centre - 0.5 * (eu + ev)
            lights.append(Light.rect(RectLight(tuple(corner), tuple(eu), tuple(ev), one_sided=True)))
        else:
            spot = Spot(axis=tuple(n), inner=math.radians(89.0), outer=math.radians(90.0))
            lights.append(Light(SphereLight(tuple(centre), float(a), spot)))
    return lights


def icosphere_field(seed: int = 2, n_spheres: int = 150, subdivisions: int = 5, width: int = 1280,
                    height: int = 720, ground_half: float = 1000.0, with_receivers: bool = True) -> Workload:
    """The plain workload at scale (about 3.07M triangles, 4 lights, 1280 x 720 hits)."""
    rng = Pcg32(seed, 22)
    meshes = [ground_quad(ground_half)]
    for i in range(n_spheres):
        r = rng.uniform(0.5, 3.0)
        cx, cz = rng.uniform(-50.0, 50.0), rng.uniform(-50.0, 50.0)
        meshes.append(displaced_icosphere((cx, r, cz), r, seed=1000 * seed + i, subdivisions=subdivisions))
    lights = icosphere_field_lights(rng)
    # A seeded azimuth around the field; 43 degrees down, so the top rows
    # still meet the ground (about 300 m away) and every pixel has a hit.
    az = 2.0 * math.pi * rng.next_f32()
    camera = np.array([75.0 * math.sin(az), 70.0, -75.0 * math.cos(az), 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 60.0],
                      np.float32)
    w = Workload("icosphere_field", meshes, np.stack([light_gpu(l) for l in lights]), None, lights, camera,
                 (width, height))
    if with_receivers:
        w.receivers = primary_hits(w, width, height)
    return w


def primary_hits(w: Workload, width: int, height: int, camera: Optional[np.ndarray] = None) -> np.ndarray:
    """Receivers at the camera's primary hits (misses dropped), via a host-only scene."""
    from .kernel import host_scene
    s = host_scene(w.meshes)
    try:
        rec, hit = s.primary_hits(camera if camera is not None else w.camera, width, height)
    finally:
        s.close()
    return np.ascontiguousarray(rec[hit.astype(bool)])


def _shape_pool(subdivisions: int, count: int, seed: int) -> list:
    """`count` unit displaced icospheres (radius 1, centred at the origin)."""
    return [displaced_icosphere((0.0, 0.0, 0.0), 1.0, seed=seed * 7919 + k, subdivisions=subdivisions)
            for k in range(count)]


def _field(rng: Pcg32, target_tris: float, pools: dict, pool: int, seed: int):
    """A field of displaced icospheres with about `target_tris` triangles on a
    ground quad; its area grows with the sphere count, so the density stays
    near icosphere_field's. Returns (meshes, half extent)."""
    sub = 5 if target_tris >= 150_000 else (4 if target_tris >= 20_000 else 3)
    per = 20 * 4 ** sub
    n = max(1, int(round((target_tris - 2) / per)))
    if sub not in pools:
        pools[sub] = _shape_pool(sub, pool, seed * 100 + sub)
    half = max(10.0, 50.0 * math.sqrt(n / 150.0))
    meshes = [ground_quad(max(1000.0, 20.0 * half))]
    for _ in range(n):
        r = rng.uniform(0.5, 3.0)
        cx, cz = rng.uniform(-half, half), rng.uniform(-half, half)
        shape = pools[sub][rng.next_u32() % pool]
        meshes.append((shape * np.float32(r) + np.array([cx, r, cz], np.float32)).astype(np.float32))
    return meshes, half


def _random_light(rng: Pcg32, half: float) -> Light:
    """A rect or disk light of size U[0.25, 4] m, 8-20 m up, tilted up to 30
    degrees from straight down, over the middle of a field."""
    h = rng.uniform(8.0, 20.0)
    x, z = rng.uniform(-0.8 * half, 0.8 * half), rng.uniform(-0.8 * half, 0.8 * half)
    nrm, u, v = _tilted_frame(rng, 30.0)
    centre = np.array([x, h, z])
    if rng.next_u32() & 1:
        eu, ev = u * rng.uniform(0.25, 4.0), v * rng.uniform(0.25, 4.0)
        if np.dot(np.cross(eu, ev), nrm) < 0:
            ev = -ev
        corner = centre - 0.5 * (eu + ev)
        return Light.rect(RectLight(tuple(corner), tuple(eu), tuple(ev), one_sided=True))
    spot = Spot(axis=tuple(nrm), inner=math.radians(89.0), outer=math.radians(90.0))
    return Light(SphereLight(tuple(centre), 0.5 * rng.uniform(0.25, 4.0), spot))


def _camera(rng: Pcg32, half: float) -> np.ndarray:
    az = 2.0 * math.pi * rng.next_f32()
    d = 1.5 * half
    return np.array([d * math.sin(az), 1.4 * half, -d * math.cos(az), 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 60.0], np.float32)


def _image(points: float):
    width = max(8, int(round(math.sqrt(points * 16.0 / 9.0))))
    return width, max(8, int(round(points / width)))


def batch_jobs(seed: int = 3, njobs: int = 64, tris=(10_000, 2_000_000), points=(4_000, 1_000_000),
               lights=(1, 16), pool: int = 16) -> list:
    """The batching workload: `njobs` jobs, each its own field of displaced
    icospheres (value-noise displacement of 0.15 r, as icosphere_field) with a
    triangle count log-uniform in `tris`, a light count uniform in `lights`
    (rects and disks of sizes U[0.25, 4] m), and the primary hits of a seeded
    camera with a point count log-uniform in `points` (misses dropped).
    Spheres are drawn from a pool of `pool` displaced shapes per subdivision
    level, scaled and placed per sphere."""
    rng = Pcg32(seed, 33)
    pools = {}
    jobs = []
    for i in range(njobs):
        t = math.exp(rng.uniform(math.log(tris[0]), math.log(tris[1])))
        meshes, half = _field(rng, t, pools, pool, seed)
        nl = lights[0] + rng.next_u32() % (lights[1] - lights[0] + 1)
        objs = [_random_light(rng, half) for _ in range(nl)]
        width, height = _image(math.exp(rng.uniform(math.log(points[0]), math.log(points[1]))))
        w = Workload(f"job{i}", meshes, np.stack([light_gpu(l) for l in objs]), None, objs, _camera(rng, half),
                     (width, height))
        w.receivers = primary_hits(w, width, height)
        jobs.append(w)
    return jobs


@dataclass
class ServedScene:
    """A resident scene of the serving workload: its meshes, its 8 base
    lights (16-float records) and the receivers of its seeded camera poses."""

    meshes: list
    lights: np.ndarray
    poses: list
    half: float = 0.0  # the field's half extent

    @property
    def ntris(self) -> int:
        return int(sum(len(m) for m in self.meshes))


def served_scenes(seed: int = 4, nscenes: int = 8, tris=(50_000, 3_000_000), poses: int = 3,
                  points=(16_000, 2_000_000), pool: int = 16) -> list:
    """The serving workload's resident scenes: `nscenes` displaced-icosphere
    fields with triangle counts log-uniform in `tris`, 8 base lights each (as
    batch_jobs'), and `poses` seeded camera poses per scene whose primary hits
    number log-uniform in `points`."""
    rng = Pcg32(seed, 44)
    pools = {}
    out = []
    for i in range(nscenes):
        t = math.exp(rng.uniform(math.log(tris[0]), math.log(tris[1])))
        meshes, half = _field(rng, t, pools, pool, seed)
        lights = np.stack([light_gpu(_random_light(rng, half)) for _ in range(8)])
        sc = ServedScene(meshes, lights, [], half)
        for _ in range(poses):
            width, height = _image(math.exp(rng.uniform(math.log(points[0]), math.log(points[1]))))
            w = Workload(f"scene{i}", meshes, lights, None, None, _camera(rng, half), (width, height))
            sc.poses.append(primary_hits(w, width, height))
        out.append(sc)
    return out


def served_requests(scenes_: list, n: int, seed: int = 5, moved: float = 0.5) -> list:
    """`n` requests over `scenes_`: (scene index, pose index, lights [k, 16])
    with k uniform in 1..8; each light is either one of the scene's base
    lights recoloured (same geometry, new radiance) or, with probability
    `moved`, a light moved to a new seeded place."""
    rng = Pcg32(seed, 55)
    reqs = []
    for _ in range(n):
        si = rng.next_u32() % len(scenes_)
        sc = scenes_[si]
        pi = rng.next_u32() % len(sc.poses)
        k = 1 + rng.next_u32() % 8
        recs = []
        for j in range(k):
            if rng.next_f32() < moved:
                recs.append(light_gpu(_random_light(rng, sc.half)))
            else:
                rec = sc.lights[(j + rng.next_u32()) % 8].copy()
                rec[12:15] = (rng.uniform(0.2, 5.0), rng.uniform(0.2, 5.0), rng.uniform(0.2, 5.0))
                recs.append(rec)
        reqs.append((si, pi, np.ascontiguousarray(np.stack(recs).astype(np.float32))))
    return reqs


def displaced_uv_sphere(seed: int, segments: int = 80, rings: int = 65, amplitude: float = 0.15,
                        frequency: float = 2.0) -> np.ndarray:
    """A unit UV sphere (segments x (2 rings - 2) triangles: 10,240 for 80 x 65)
    with vertices moved radially by seeded value noise of amplitude
    `amplitude`, centred at the origin, +Z poles, outward winding."""
    base = sphere_mesh((0.0, 0.0, 0.0), 1.0, segments, rings).astype(np.float64)
    flat = base.reshape(-1, 3)
    unit = flat / np.linalg.norm(flat, axis=1, keepdims=True)
    scale = 1.0 + amplitude * value_noise(unit * frequency, seed)
    return (unit * scale[:, None]).reshape(-1, 3, 3).astype(np.float32)


@dataclass
class InstancedWorld:
    """Shared geometries (object space), cc_instance records placing them, lights
    and receivers."""

    geometries: list
    instances: np.ndarray
    lights: np.ndarray
    receivers: Optional[np.ndarray] = None
    camera: Optional[np.ndarray] = None
    size: Optional[tuple] = None

    @property
    def instanced_tris(self) -> int:
        counts = np.array([len(g) for g in self.geometries])
        return int(counts[self.instances["geometry"]].sum())


def yaw_rotation(angle: float) -> np.ndarray:
    """Rotation about +Y by `angle`, row-major."""
    c, s = math.cos(angle), math.sin(angle)
    return np.array([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]], np.float32)


def instanced_world(seed: int = 5, n_instances: int = 1_000_000, n_boulders: int = 10, half: float = 2000.0,
                    n_lights: int = 8, width: int = 1280, height: int = 720, segments: int = 80, rings: int = 65,
                    with_receivers: bool = True) -> InstancedWorld:
    """The instanced large world: `n_boulders` displaced UV-sphere boulders
    (10,240 triangles each at 80 x 65) placed as `n_instances` instances with
    scale U[0.5, 4], yaw U[0, 2 pi] and positions U[-half, half]^2 resting on a
    ground quad (itself one more instance); `n_lights` rect and disk lights
    (as batch_jobs') over the camera's view; the primary hits of a seeded
    camera (misses dropped)."""
    rng = Pcg32(seed, 66)
    geometries = [displaced_uv_sphere(seed * 100 + k, segments, rings) for k in range(n_boulders)]
    geometries.append(ground_quad(1.0))
    ground = len(geometries) - 1
    inst = np.zeros(n_instances + 1, _lib_instance_dtype())
    eye_r = np.random.default_rng(seed)  # placements: vectorized, seeded
    g = eye_r.integers(0, n_boulders, n_instances)
    scale = eye_r.uniform(0.5, 4.0, n_instances).astype(np.float32)
    yaw = eye_r.uniform(0.0, 2.0 * math.pi, n_instances)
    x = eye_r.uniform(-half, half, n_instances).astype(np.float32)
    z = eye_r.uniform(-half, half, n_instances).astype(np.float32)
    c, s = np.cos(yaw).astype(np.float32), np.sin(yaw).astype(np.float32)
    rot = np.zeros((n_instances, 9), np.float32)
    rot[:, 0], rot[:, 2], rot[:, 4], rot[:, 6], rot[:, 8] = c, s, 1.0, -s, c
    inst["geometry"][:n_instances] = g
    inst["rotation"][:n_instances] = rot
    inst["scale"][:n_instances] = scale
    inst["translation"][:n_instances] = np.stack([x, scale, z], 1)
    inst[n_instances] = (ground, np.eye(3, dtype=np.float32).reshape(9), half * 1.05, (0.0, 0.0, 0.0))
    # The camera looks at a seeded spot; the lights hang over what it sees.
    cx, cz = rng.uniform(-0.5 * half, 0.5 * half), rng.uniform(-0.5 * half, 0.5 * half)
    az = 2.0 * math.pi * rng.next_f32()
    camera = np.array([cx + 60.0 * math.sin(az), 35.0, cz - 60.0 * math.cos(az), cx, 0.0, cz, 0.0, 1.0, 0.0, 60.0],
                      np.float32)
    objs = []
    for _ in range(n_lights):
        l = _random_light(rng, 40.0)
        objs.append(l)
    lights = np.stack([light_gpu(l) for l in objs])
    lights[:, 0] += cx  # over the view (corner / centre x and z)
    lights[:, 2] += cz
    w = InstancedWorld(geometries, inst, lights, None, camera, (width, height))
    if with_receivers:
        from .kernel import host_scene_instanced
        hs = host_scene_instanced(geometries, inst)
        try:
            rec, hit = hs.primary_hits(camera, width, height)
        finally:
            hs.close()
        w.receivers = np.ascontiguousarray(rec[hit.astype(bool)])
    return w


def _lib_instance_dtype():
    from ._lib import INSTANCE_DTYPE
    return INSTANCE_DTYPE


def moved_placements(world: InstancedWorld, movable: np.ndarray, frame: int, step: float = 3.0) -> np.ndarray:
    """New cc_instance records for the movable objects (in their order) at
    `frame`: each moved by a seeded offset of up to `step` metres in x and z
    and turned by a seeded yaw; geometry and scale kept."""
    rng = np.random.default_rng(10_000 + frame)
    base = world.instances[np.asarray(movable)]
    out = base.copy()
    n = len(out)
    off = rng.uniform(-step, step, (n, 2)).astype(np.float32) * np.float32(frame)
    out["translation"][:, 0] += off[:, 0]
    out["translation"][:, 2] += off[:, 1]
    yaw = rng.uniform(0.0, 2.0 * math.pi, n)
    c, s = np.cos(yaw).astype(np.float32), np.sin(yaw).astype(np.float32)
    rot = np.zeros((n, 9), np.float32)
    rot[:, 0], rot[:, 2], rot[:, 4], rot[:, 6], rot[:, 8] = c, s, 1.0, -s, c
    out["rotation"] = rot
    return out


def grid_pages(grid: np.ndarray, surface: Optional[np.ndarray] = None, object_id: int = 0) -> list:
    """Lighting-cache pages over a (rows, cols) grid of receivers, a stand-in
    for one chart at one mip (the cache's charts are not part of this
    library): page (px, py) holds the grid points [py * 8 + y, px * 8 + x]
    for x, y in 0..8 (8 x 8 texels stored 9 x 9, vcache.rs:32-35); `inside`
    counts those within the grid; a texel's flag is 2 where `surface` is true
    (all by default), 1 where it is not, 0 past the grid; the grid's own
    triangles (normal.w, as the camera pass writes them) are kept. Keys are
    (object_id, py, px); priorities 0."""
    from .kernel import PageRequest
    rows, cols = grid.shape[:2]
    if surface is None:
        surface = np.ones((rows, cols), bool)
    pages = []
    for py in range((rows - 1) // 8 + 1 if rows > 1 else 1):
        for px in range((cols - 1) // 8 + 1 if cols > 1 else 1):
            t = np.zeros((9, 9, 8), np.float32)
            r0, c0 = py * 8, px * 8
            ins = (min(9, cols - c0), min(9, rows - r0))
            t[: ins[1], : ins[0]] = grid[r0:r0 + ins[1], c0:c0 + ins[0]]
            t[: ins[1], : ins[0], 3] = np.where(surface[r0:r0 + ins[1], c0:c0 + ins[0]], 2.0, 1.0)
            pages.append(PageRequest((object_id, py, px), 0, ins, t.reshape(81, 8)))
    return pages
