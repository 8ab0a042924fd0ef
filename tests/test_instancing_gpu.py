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


def test_moved_objects_mark_the_oracle_stale_cones_and_the_update_equals_a_full_solve(kernel, world):
    """Move every tenth boulder; the device's stale cones are the oracle's,
    the incremental update leaves every uncapped cone as a full solve of the
    moved scene gives it, and the moved scene meets the parity bar."""
    import torch

    from continuum_b200 import _lib

    movable = np.arange(0, len(world.instances) - 1, 10, dtype=np.uint32)
    scene = kernel.scene_instanced(world.geometries, world.instances, movable)
    orc = OracleScene.instanced(world.geometries, world.instances, movable)
    dev = torch.device("cuda:0")
    rec = torch.from_numpy(world.receivers).to(dev)
    lig = torch.from_numpy(world.lights).to(dev)
    P, L = rec.shape[0], lig.shape[0]
    n = P * L
    cache = {"full": torch.zeros(n, dtype=torch.int64, device=dev), "any": torch.zeros(n, dtype=torch.int64, device=dev),
             "irradiance": torch.zeros(n, device=dev), "fraction": torch.zeros(n, device=dev)}
    ptrs = {k: v.data_ptr() for k, v in cache.items()}
    kernel.visibility_device(scene, rec.data_ptr(), P, lig.data_ptr(), L, ptrs)
    torch.cuda.synchronize()

    pl = scenes.moved_placements(world, movable, 1)
    boxes = scene.move(pl)
    assert np.array_equal(boxes, orc.move(pl))
    stale = torch.zeros(n, dtype=torch.uint8, device=dev)
    count = kernel.stale_cones(scene, rec.data_ptr(), P, world.lights, boxes, stale.data_ptr())
    want = orc.stale_cones(world.receivers, world.lights, boxes)
    assert np.array_equal(stale.cpu().numpy(), want)
    assert count == int(want.sum()) and 0 < count < n

    solved = kernel.visibility_update(scene, rec.data_ptr(), P, lig.data_ptr(), L, stale.data_ptr(), ptrs)
    assert solved == count
    full = parity.flat(kernel.visibility(scene, world.receivers, world.lights, outputs=ALL))
    capped = (full["work"][:, 3] & _lib.CC_CONE_CAPPED) != 0
    got = {k: v.cpu().numpy() for k, v in cache.items()}
    for k in ("full", "any", "irradiance", "fraction"):
        a, b = got[k].reshape(-1), np.asarray(full[k]).reshape(-1)
        if k in ("full", "any"):
            a = a.view(np.uint64)
        assert np.array_equal(a[~capped], b[~capped]), k
    o = orc.visibility(world.receivers, world.lights)
    parity.compare(full, o, o["unshadowed"])
    scene.close()
    orc.close()


def test_update_in_small_chunks_equals_the_default(kernel, world):
    """The incremental update walks its listed cones a chunk at a time; small
    chunks give the same cache as the default."""
    import torch

    movable = np.arange(0, len(world.instances) - 1, 10, dtype=np.uint32)
    scene = kernel.scene_instanced(world.geometries, world.instances, movable)
    dev = torch.device("cuda:0")
    rec = torch.from_numpy(world.receivers).to(dev)
    lig = torch.from_numpy(world.lights).to(dev)
    P, L = rec.shape[0], lig.shape[0]
    n = P * L

    def cache():
        return {"full": torch.zeros(n, dtype=torch.int64, device=dev), "any": torch.zeros(n, dtype=torch.int64, device=dev),
                "irradiance": torch.zeros(n, device=dev), "fraction": torch.zeros(n, device=dev)}

    caches = [cache(), cache()]
    for c in caches:
        kernel.visibility_device(scene, rec.data_ptr(), P, lig.data_ptr(), L, {k: v.data_ptr() for k, v in c.items()})
    torch.cuda.synchronize()
    boxes = scene.move(scenes.moved_placements(world, movable, 1))
    stale = torch.zeros(n, dtype=torch.uint8, device=dev)
    count = kernel.stale_cones(scene, rec.data_ptr(), P, world.lights, boxes, stale.data_ptr())
    assert count > 1000
    try:
        for c, chunk in zip(caches, (1 << 25, 1000)):
            kernel.set_split_chunk(chunk)
            solved = kernel.visibility_update(scene, rec.data_ptr(), P, lig.data_ptr(), L, stale.data_ptr(),
                                              {k: v.data_ptr() for k, v in c.items()})
            assert solved == count
        torch.cuda.synchronize()
        for k in caches[0]:
            assert torch.equal(caches[0][k], caches[1][k]), k
    finally:
        kernel.set_split_chunk(1 << 25)
        scene.close()


def clear_values(world):
    """Some boulders alpha-blended (clear 0.5), some thin glass (-0.7), some
    solid glass volumes (-2.5); the ground stays opaque."""
    clear = np.zeros(len(world.instances), np.float32)
    clear[0:-1:7] = 0.5
    clear[3:-1:11] = -0.7
    clear[5:-1:13] = -2.5
    return clear


def test_blended_and_transmissive_objects_match_the_oracle(kernel, world):
    """Placed objects' `clear` (Placement::clear; add_mesh_coverage_if and
    cover_triangle, mask_cones.wgsl:600-614, :725-741): blended objects'
    triangles drawn with 1 - clear, transmissive ones with one less the
    Fresnel-weighted share passing through, against the oracle at the parity
    bar; their shadows let light through where opaque ones would not."""
    clear = clear_values(world)
    scene = kernel.scene_instanced(world.geometries, world.instances)
    opaque = parity.flat(kernel.visibility(scene, world.receivers, world.lights, outputs=ALL))
    scene.set_clear(clear)
    g = parity.flat(kernel.visibility(scene, world.receivers, world.lights, outputs=ALL))
    scene.close()
    orc = OracleScene.instanced(world.geometries, world.instances)
    orc.set_clear(clear)
    o = orc.visibility(world.receivers, world.lights)
    orc.close()
    parity.compare(g, o, o["unshadowed"])
    lit = g["fraction"] > opaque["fraction"] + 1e-3
    assert lit.sum() > 50
    assert np.all(g["fraction"] >= opaque["fraction"] - 1e-6)


def test_prefiltered_cones_through_blended_objects_match_the_oracle(kernel, world):
    """At 8 bins some nodes of this world are splatted (their coverage samples
    scaled by their geometry's opacity): the results differ from exact cones
    and meet the bar against the oracle's prefiltered walk."""
    clear = clear_values(world)
    scene = kernel.scene_instanced(world.geometries, world.instances)
    scene.set_clear(clear)
    exact = parity.flat(kernel.visibility(scene, world.receivers, world.lights, outputs=ALL))
    kernel.prefilter = 8.0
    try:
        g = parity.flat(kernel.visibility(scene, world.receivers, world.lights, outputs=ALL))
    finally:
        kernel.prefilter = 0.0
        scene.close()
    assert (g["fraction"] != exact["fraction"]).sum() > 10
    orc = OracleScene.instanced(world.geometries, world.instances)
    orc.set_clear(clear)
    o = orc.visibility(world.receivers, world.lights, prefilter=8.0)
    orc.close()
    parity.compare(g, o, o["unshadowed"])
