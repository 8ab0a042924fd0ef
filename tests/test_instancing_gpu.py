"""Instanced scenes on a B200: cones walked into each placed object's space
(cone_to_object, mask_cones.wgsl:623-638) against the oracle's restatement,
for every hierarchy mode."""
import numpy as np
import pytest

import parity
from continuum_b200 import scenes
from oracle.oracle import OracleScene

pytestmark = pytest.mark.gpu

ALL = ("full", "any", "partial", "irradiance", "fraction", "work")


@pytest.fixture(scope="module")
def world():
    return scenes.instanced_world(seed=3, n_instances=300, n_boulders=3, half=40.0, n_lights=4, width=96, height=54,
                                  segments=24, rings=13)


@pytest.mark.parametrize("hierarchy,points", [(2, None), (1, 2048), (0, 256)])
def test_instanced_world_matches_the_oracle(kernel, world, hierarchy, points):
    rec = world.receivers if points is None else np.ascontiguousarray(world.receivers[:: max(1, world.receivers.shape[0] // points)][:points])
    scene = kernel.scene_instanced(world.geometries, world.instances)
    g = parity.flat(kernel.visibility(scene, rec, world.lights, hierarchy=hierarchy, outputs=ALL))
    scene.close()
    orc = OracleScene.instanced(world.geometries, world.instances)
    o = orc.visibility(rec, world.lights, hierarchy=hierarchy)
    orc.close()
    stats = parity.compare(g, o, o["unshadowed"])
    assert stats["cones"] == rec.shape[0] * world.lights.shape[0]
    # The boulders cast shadows: some cones are covered.
    assert (g["any"] != 0).mean() > 0.01


def test_instanced_packets_equal_solo_walks(kernel, world):
    scene = kernel.scene_instanced(world.geometries, world.instances)
    runs = [parity.flat(kernel.visibility(scene, world.receivers, world.lights, outputs=ALL, points_per_warp=p))
            for p in (1, 32)]
    scene.close()
    for k in ("full", "any", "partial", "irradiance", "fraction"):
        assert np.array_equal(runs[0][k], runs[1][k]), k
