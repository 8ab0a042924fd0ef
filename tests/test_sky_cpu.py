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
