"""Prefiltered cones on a B200 (cc_options.prefilter) against the oracle's
prefiltered walk: light cones within the parity bar, sky cones within the
sky bar (tests/test_sky_gpu.py), plain and instanced scenes, object-level
splats on and off, and packets equal to solo walks."""
import math

import numpy as np
import pytest

import parity
from continuum_b200 import _lib, scenes
from oracle.oracle import SUM_FIXED, OracleScene

pytestmark = pytest.mark.gpu
ALL = ("full", "any", "partial", "irradiance", "fraction", "work")


@pytest.fixture(scope="module")
def field():
    return scenes.icosphere_field(seed=5, n_spheres=12, subdivisions=4, width=96, height=54)


@pytest.fixture(scope="module")
def world():
    return scenes.instanced_world(seed=3, n_instances=300, n_boulders=3, half=40.0, n_lights=4, width=96, height=54,
                                  segments=24, rings=18)


def light_parity(kernel, scene, orc, rec, lights, prefilter, object_prefilter=True, ppw=None):
    kernel.prefilter, kernel.object_prefilter = prefilter, object_prefilter
    try:
        g = parity.flat(kernel.visibility(scene, rec, lights, outputs=ALL, points_per_warp=ppw))
    finally:
        kernel.prefilter, kernel.object_prefilter = 0.0, True
    o = orc.visibility(rec, lights, prefilter=prefilter, object_prefilter=object_prefilter)
    parity.compare(g, o, o["unshadowed"])
    return g, o


@pytest.mark.parametrize("prefilter", [1.0, 4.0])
def test_prefiltered_light_cones(kernel, field, prefilter):
    scene = kernel.scene(field.meshes)
    try:
        light_parity(kernel, scene, OracleScene(field.meshes), field.receivers, field.lights, prefilter)
    finally:
        scene.close()


@pytest.mark.parametrize("object_prefilter", [True, False])
def test_prefiltered_instanced_light_cones(kernel, world, object_prefilter):
    scene = kernel.scene_instanced(world.geometries, world.instances)
    try:
        light_parity(kernel, scene, OracleScene.instanced(world.geometries, world.instances), world.receivers,
                     world.lights, 2.0, object_prefilter)
    finally:
        scene.close()


def test_prefiltered_packets_equal_solo_walks(kernel, field):
    scene = kernel.scene(field.meshes)
    kernel.prefilter = 2.0
    try:
        runs = [parity.flat(kernel.visibility(scene, field.receivers, field.lights, outputs=ALL, points_per_warp=p))
                for p in (32, 1)]
    finally:
        kernel.prefilter = 0.0
        scene.close()
    for k in ("full", "any", "partial", "irradiance", "fraction"):
        assert np.array_equal(runs[0][k], runs[1][k]), k


def sky_parity(kernel, scene, orc, rec, prefilter, object_prefilter=True, agreement=0.99):
    kernel.prefilter, kernel.object_prefilter = prefilter, object_prefilter
    try:
        irr, faces = kernel.sky_visibility(scene, rec, outputs=("full", "any", "partial", "irradiance"))
    finally:
        kernel.prefilter, kernel.object_prefilter = 0.0, True
    g = {"full": faces.full.reshape(-1), "any": faces.any.reshape(-1), "partial": faces.partial.reshape(-1, 64)}
    # The light cones' bar against the oracle with the library's summation;
    # against the reference's walk-order f32 sums, `agreement` (see
    # tests/test_sky_gpu.py), every disagreeing bit traced either way.
    fixed = orc.sky_visibility(rec, prefilter=prefilter, flags=0 if object_prefilter else 4, accumulate=SUM_FIXED)
    stats = parity.compare(g, fixed, None, check=False)
    assert stats["untraced_bits"] == 0, stats
    assert stats["word_agreement"] >= parity.WORD_AGREEMENT, stats
    o = orc.sky_visibility(rec, prefilter=prefilter, flags=0 if object_prefilter else 4)
    stats = parity.compare(g, o, None, check=False)
    assert stats["untraced_bits"] == 0, stats
    assert stats["word_agreement"] >= agreement, stats
    assert np.abs(faces.irradiance.reshape(-1) - o["face_light"]).max() <= 2e-3 * math.pi
    assert np.abs(irr - o["irradiance"]).max() <= 2e-3 * math.pi


def test_prefiltered_sky_cones(kernel, field):
    scene = kernel.scene(field.meshes)
    try:
        sky_parity(kernel, scene, OracleScene(field.meshes), field.receivers, 1.0)
    finally:
        scene.close()


@pytest.mark.parametrize("object_prefilter", [True, False])
def test_prefiltered_instanced_sky_cones(kernel, world, object_prefilter):
    rec = np.ascontiguousarray(world.receivers[::3])
    scene = kernel.scene_instanced(world.geometries, world.instances)
    try:
        # Against the reference's summation, splats of many small nodes
        # combined as independent occluders leave more bins within its
        # rounding of whole: 97.4 % of face cones agree word for word here,
        # every other bit traced.
        sky_parity(kernel, scene, OracleScene.instanced(world.geometries, world.instances), rec, 1.0, object_prefilter,
                   agreement=0.95)
    finally:
        scene.close()


def test_prefilter_needs_the_triangle_hierarchy(kernel, field):
    scene = kernel.scene(field.meshes)
    kernel.prefilter = 1.0
    try:
        with pytest.raises(_lib.CCError):
            kernel.visibility(scene, field.receivers[:64], field.lights, hierarchy=1)
    finally:
        kernel.prefilter = 0.0
        scene.close()
