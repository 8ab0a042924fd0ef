"""Sky cones in the oracle (mask_cones.wgsl:1323-1511): known answers that
pin the restatement before it checks the library."""
import math

import numpy as np

import kat
from continuum_b200 import scenes
from oracle.oracle import OracleScene


def ground_receivers(normals, y=1e-4):
    n = np.asarray(normals, np.float64)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    pts = np.zeros((len(n), 3))
    pts[:, 1] = y
    pts[:, 0] = np.linspace(-3, 3, len(n))
    return kat.receivers(pts.astype(np.float32), n.astype(np.float32))


def test_open_sky_is_pi_for_any_normal():
    """Nothing above the horizon: the six faces' clipped windows tile the
    hemisphere, so the irradiance per unit sky radiance is pi (cosine-weighted
    hemisphere) whatever the normal; the only geometry lies below every
    receiver's tangent plane and is skipped."""
    rng = np.random.default_rng(4)
    normals = rng.normal(size=(64, 3))
    normals[:, 1] = np.abs(normals[:, 1]) + 0.3
    below = scenes.box_mesh((-1.0, -1e4, -1.0), (1.0, -1e4 + 1.0, 1.0))
    o = OracleScene([below])
    for precision, tol in ((8, 1e-7), (4, 2e-5)):  # results are returned as f32
        r = o.sky_visibility(ground_receivers(normals), precision=precision)
        assert np.abs(r["irradiance"] - math.pi).max() <= tol * math.pi, np.abs(r["irradiance"] - math.pi).max()


def test_a_roof_blocks_the_sky_and_walls_block_their_share():
    """Under a large roof the sky is (nearly) gone; beside a wall half the
    sky's share toward it is gone, as the FP64 oracle finds it."""
    rec = ground_receivers([[0, 1, 0]] * 4)
    roof = scenes.box_mesh((-500.0, 2.0, -500.0), (500.0, 2.1, 500.0))
    r = OracleScene([scenes.ground_quad(50.0), roof]).sky_visibility(rec, precision=8)
    assert np.all(r["irradiance"] < 0.01 * math.pi)
    wall = scenes.box_mesh((5.0, 0.0, -500.0), (5.1, 500.0, 500.0))
    r = OracleScene([scenes.ground_quad(50.0), wall]).sky_visibility(rec, precision=8)
    assert np.all(r["irradiance"] < 0.999 * math.pi) and np.all(r["irradiance"] > 0.5 * math.pi)


def test_float_matches_double_and_flags_change_what_they_should():
    w = scenes.box_field(grid=24)
    o = OracleScene(w.meshes)
    r32 = o.sky_visibility(w.receivers)
    r64 = o.sky_visibility(w.receivers, precision=8)
    assert np.abs(r32["irradiance"] - r64["irradiance"]).max() <= 1e-5 * math.pi
    rmax = o.sky_visibility(w.receivers, flags=1)
    # Independent occluders block at least as much as the maximum.
    assert np.all(rmax["irradiance"] >= r32["irradiance"] - 1e-6)
    assert np.any(rmax["irradiance"] > r32["irradiance"] + 1e-6)
    # Faces wholly below the horizon (the -y face of an upward normal) see nothing.
    face_light = r32["face_light"].reshape(6, -1)
    assert np.all(face_light[3] == 0.0)
    assert np.allclose(face_light.sum(0), r32["irradiance"], atol=1e-5)


def test_open_sky_is_pi_in_any_objects_frame():
    """Faces turned with the receiver's object (flag 8: sky_frame,
    mask_cones.wgsl:1432-1456) still tile the hemisphere: a uniform open sky
    gives pi whatever the object's rotation; the turned faces see a wall
    differently from world-axis faces, but their light sums to the same
    total where nothing blocks it."""
    from continuum_b200._lib import INSTANCE_DTYPE

    rng = np.random.default_rng(6)
    geo = [scenes.box_mesh((-1.0, -1.0, -1.0), (1.0, 1.0, 1.0))]
    inst = np.zeros(5, INSTANCE_DTYPE)
    for i in range(5):
        a = rng.normal(size=3)
        a /= np.linalg.norm(a)
        ang = rng.uniform(0, 2 * math.pi)
        k = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
        rot = np.eye(3) + math.sin(ang) * k + (1 - math.cos(ang)) * k @ k  # Rodrigues
        inst[i] = (0, rot.astype(np.float32).reshape(9), 1.0, (i * 10.0, -1e4, 0.0))
    o = OracleScene.instanced(geo, inst)
    normals = rng.normal(size=(40, 3))
    normals[:, 1] = np.abs(normals[:, 1]) + 0.3
    rec = ground_receivers(normals)
    rec[:, 3] = (np.arange(40, dtype=np.uint32) % 5).view(np.float32)  # the object each receiver lies on
    for precision, tol in ((8, 1e-7), (4, 2e-5)):
        framed = o.sky_visibility(rec, precision=precision, flags=8)
        assert np.abs(framed["irradiance"] - math.pi).max() <= tol * math.pi
    world = o.sky_visibility(rec, precision=8)
    framed = o.sky_visibility(rec, precision=8, flags=8)
    assert not np.allclose(world["face_light"], framed["face_light"])  # the faces did turn
    o.close()
