"""Sky cones on a B200 (cc_sky_visibility) against the oracle: per face cone
the FULL/ANY words and coverage, per face and per receiver the light within
2e-3 of the open sky's (pi); the open sky is pi.

Mask words are held to the light cones' bar (99.9 % of face cones word for
word, every disagreeing bit traced to coverage within 2e-5 of whole or of
nothing on both sides) against the oracle summing each mesh's cells as the
library does (fixed point, 2^-24 of a bin per add). Against the oracle
summing in walk order in f32, as the reference does, every disagreeing bit
is traced the same way and at least 99 % of face cones agree: a face's
window is 90 degrees wide and reaches past the whole scene, so far more bins
end within the reference's rounding of whole or of nothing than a light
cone's do."""
import math

import numpy as np
import pytest

import kat
import parity
from continuum_b200 import _lib, scenes
from oracle.oracle import SUM_FIXED, OracleScene

pytestmark = pytest.mark.gpu
SKY_TOL = 2e-3 * math.pi


def oracle_flags(sky_flags):
    """The oracle's sky flags for cc_sky_visibility's."""
    return ((1 if sky_flags & _lib.CC_SKY_COMBINE_MAX else 0) | (2 if sky_flags & _lib.CC_SKY_NO_HORIZON_CULL else 0) |
            (8 if sky_flags & _lib.CC_SKY_OBJECT_FRAME else 0))


def check_against_oracle(kernel, meshes, rec, sky_flags=0, instanced=None):
    scene = kernel.scene(meshes) if instanced is None else kernel.scene_instanced(*instanced)
    try:
        irr, faces = kernel.sky_visibility(scene, rec, sky_flags=sky_flags,
                                           outputs=("full", "any", "partial", "irradiance", "work"))
    finally:
        scene.close()
    orc = OracleScene(meshes) if instanced is None else OracleScene.instanced(*instanced)
    g = {"full": faces.full.reshape(-1), "any": faces.any.reshape(-1), "partial": faces.partial.reshape(-1, 64)}
    fixed = orc.sky_visibility(rec, flags=oracle_flags(sky_flags), accumulate=SUM_FIXED)
    stats = parity.compare(g, fixed, None, check=False)
    assert stats["untraced_bits"] == 0, stats
    assert stats["word_agreement"] >= parity.WORD_AGREEMENT, stats
    o = orc.sky_visibility(rec, flags=oracle_flags(sky_flags))
    walk = parity.compare(g, o, None, check=False)
    assert walk["untraced_bits"] == 0, walk
    assert walk["word_agreement"] >= 0.99, walk
    assert np.abs(faces.irradiance.reshape(-1) - o["face_light"]).max() <= SKY_TOL
    assert np.abs(irr - o["irradiance"]).max() <= SKY_TOL
    # The per-receiver sum is the faces' light summed in face order.
    f = faces.irradiance.reshape(6, -1)
    total = np.zeros(f.shape[1], np.float32)
    for k in range(6):
        total = (total + f[k]).astype(np.float32)
    assert np.array_equal(total, irr)
    return irr, faces, o, stats


def test_sky_box_field(kernel):
    w = scenes.box_field(grid=64)
    rec = w.receivers.copy()
    rec[:, 1] = 1e-4  # lifted off the ground as surface_offset does
    irr, faces, o, stats = check_against_oracle(kernel, w.meshes, rec)
    assert stats["cones"] == 6 * rec.shape[0]
    assert irr.min() < 0.99 * math.pi  # the boxes block some sky


@pytest.mark.parametrize("flags", [_lib.CC_SKY_COMBINE_MAX, _lib.CC_SKY_NO_HORIZON_CULL])
def test_sky_flags(kernel, flags):
    w = scenes.box_field(grid=32)
    rec = w.receivers.copy()
    rec[:, 1] = 1e-4
    check_against_oracle(kernel, w.meshes, rec, sky_flags=flags)


@pytest.mark.parametrize("flags", [0, _lib.CC_SKY_COMBINE_MAX])
def test_sky_icosphere_field(kernel, flags):
    f = scenes.icosphere_field(seed=5, n_spheres=12, subdivisions=4, width=96, height=54)
    check_against_oracle(kernel, f.meshes, f.receivers, sky_flags=flags)


def test_open_sky_is_pi(kernel):
    rng = np.random.default_rng(4)
    n = rng.normal(size=(2048, 3))
    n[:, 1] = np.abs(n[:, 1]) + 0.3
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    pts = np.zeros((2048, 3), np.float32)
    pts[:, 0] = np.linspace(-3, 3, 2048)
    rec = kat.receivers(pts, n.astype(np.float32))
    below = scenes.box_mesh((-1.0, -1e4, -1.0), (1.0, -1e4 + 1.0, 1.0))
    scene = kernel.scene([below])
    try:
        irr, _ = kernel.sky_visibility(scene, rec)
    finally:
        scene.close()
    assert np.abs(irr - math.pi).max() <= 2e-5 * math.pi


def test_sky_device_pointers(kernel):
    import torch
    w = scenes.box_field(grid=32)
    rec = w.receivers.copy()
    rec[:, 1] = 1e-4
    scene = kernel.scene(w.meshes)
    try:
        host, _ = kernel.sky_visibility(scene, rec)
        dev = torch.device("cuda:0")
        r = torch.from_numpy(rec).to(dev)
        out = torch.zeros(rec.shape[0], device=dev)
        faces = torch.zeros(6 * rec.shape[0], device=dev)
        kernel.sky_visibility_device(scene, r.data_ptr(), rec.shape[0], out.data_ptr(),
                                     faces={"irradiance": faces.data_ptr()})
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), host)
    finally:
        scene.close()


def test_sky_instanced_world(kernel):
    """Sky cones walked into each object's space (the horizon turns with the
    cone, cone_to_object :634)."""
    w = scenes.instanced_world(seed=3, n_instances=300, n_boulders=3, half=40.0, n_lights=4, width=96, height=54,
                               segments=24, rings=18)
    rec = np.ascontiguousarray(w.receivers[::3])
    check_against_oracle(kernel, None, rec, instanced=(w.geometries, w.instances))


def receivers_on_objects(w, count, seed=7):
    """Receivers on the boulders of an instanced world: a triangle's centroid
    of a random instance, placed and lifted 1e-3 along its world normal, with
    the instance's index in point.w (as bits) for CC_SKY_OBJECT_FRAME."""
    rng = np.random.default_rng(seed)
    inst = w.instances
    rec = np.zeros((count, 8), np.float32)
    objects = rng.integers(0, len(inst) - 1, count)  # the last instance is the ground
    for i, m in enumerate(objects):
        g = w.geometries[inst["geometry"][m]].reshape(-1, 3, 3).astype(np.float64)
        t = g[rng.integers(0, len(g))]
        rot = inst["rotation"][m].reshape(3, 3).astype(np.float64)
        c = rot @ t.mean(axis=0) * inst["scale"][m] + inst["translation"][m]
        n = rot @ np.cross(t[1] - t[0], t[2] - t[0])
        n /= np.linalg.norm(n)
        rec[i, 0:3] = c + n * 1e-3 * inst["scale"][m]
        rec[i, 4:7] = n
    rec[:, 3] = objects.astype(np.uint32).view(np.float32)
    rec[-4:, 3] = np.array([0xFFFFFFFF] * 4, np.uint32).view(np.float32)  # world axes
    return rec


def test_sky_faces_in_the_receivers_object_frame(kernel):
    """CC_SKY_OBJECT_FRAME (the reference's sky_frame, set_sky_object_frame):
    each receiver's cube of faces turns with the object it lies on. Against
    the oracle, and different from world axes where the objects are turned."""
    w = scenes.instanced_world(seed=3, n_instances=300, n_boulders=3, half=40.0, n_lights=4, width=96, height=54,
                               segments=24, rings=18)
    rec = receivers_on_objects(w, 1024)
    irr, faces, o, stats = check_against_oracle(kernel, None, rec, sky_flags=_lib.CC_SKY_OBJECT_FRAME,
                                                instanced=(w.geometries, w.instances))
    assert stats["cones"] == 6 * 1024
    scene = kernel.scene_instanced(w.geometries, w.instances)
    try:
        world_irr, world_faces = kernel.sky_visibility(scene, rec, outputs=("full",))
    finally:
        scene.close()
    # Receivers on turned objects see their faces' masks change; NONE keeps world axes.
    assert (world_faces.full.reshape(6, -1)[:, :-4] != faces.full.reshape(6, -1)[:, :-4]).any()
    assert np.array_equal(world_faces.full.reshape(6, -1)[:, -4:], faces.full.reshape(6, -1)[:, -4:])
