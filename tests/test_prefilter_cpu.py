"""Prefiltered cones on the host: the library's coverage samples (27 per
node, hierarchy.rs:546-569, :661-707) equal the oracle's restatement bit for
bit, and the oracle's prefiltered walk behaves as the reference describes."""
import math

import numpy as np

from continuum_b200 import host_scene, host_scene_instanced, scenes
from oracle.oracle import OracleScene


def test_triangle_node_coverage_matches_the_oracle():
    f = scenes.icosphere_field(seed=5, n_spheres=12, subdivisions=3, width=16, height=9)
    lib = host_scene(f.meshes)
    try:
        blas, obj = lib.coverage()
        sphere_root = int(lib.arrays()["ranges"][1, 2])
    finally:
        lib.close()
    ob, oo = OracleScene(f.meshes).coverage()
    assert obj is None and oo is None
    assert blas.shape == ob.shape and np.array_equal(blas, ob)
    # A closed mesh (a displaced sphere) shows its front area from every
    # direction, about the same from opposite ones.
    root = blas[sphere_root]
    assert np.all(root[:13] > 0)
    assert np.allclose(root[:13], root[14:][::-1], rtol=1e-3)


def test_object_node_coverage_matches_the_oracle():
    w = scenes.instanced_world(seed=3, n_instances=200, n_boulders=3, half=40.0, n_lights=2, width=16, height=9,
                               segments=16, rings=12, with_receivers=False)
    movable = np.arange(0, 200, 10, dtype=np.uint32)
    lib = host_scene_instanced(w.geometries, w.instances, movable)
    try:
        blas, obj = lib.coverage()
    finally:
        lib.close()
    ob, oo = OracleScene.instanced(w.geometries, w.instances, movable).coverage()
    assert np.array_equal(blas, ob)
    # The library flags nodes without prefiltered coverage in sample 13 (the
    # root over movers and the movers' subtree); the oracle reads info.z.
    flagged = obj[:, 13] == 1.0
    assert flagged[0] and flagged[2] and not flagged[1]
    obj_cmp = obj.copy()
    obj_cmp[:, 13] = 0.0
    assert np.array_equal(obj_cmp, oo)


def test_blended_and_transmissive_objects_scale_their_geometry_coverage():
    """flatten_instanced (hierarchy.rs:469-503): a geometry's node samples
    scale by the opacity of the first object placing it (blended: 1 - clear;
    transmissive: 1 - 0.96 (-clear); a volume: 1 - (0.96 (-2 - clear))^2),
    in the library as in the oracle; a move keeps each object's clear."""
    w = scenes.instanced_world(seed=3, n_instances=200, n_boulders=3, half=40.0, n_lights=2, width=16, height=9,
                               segments=16, rings=12, with_receivers=False)
    movable = np.arange(0, 200, 10, dtype=np.uint32)
    clear = np.zeros(len(w.instances), np.float32)
    first = {}
    for k, inst in enumerate(w.instances):
        first.setdefault(int(inst["geometry"]), k)
    g_of = sorted(first)
    clear[first[g_of[0]]] = 0.5
    clear[first[g_of[1]]] = -0.6
    clear[first[g_of[2]]] = -2.4
    clear[first[g_of[0]] + 1] = 0.25  # not the geometry's first object: no effect on its samples
    lib = host_scene_instanced(w.geometries, w.instances, movable)
    base, _ = lib.coverage()
    lib.set_clear(clear)
    try:
        blas, obj = lib.coverage()
        assert not np.array_equal(blas, base)
        xf = lib.transforms()
        assert np.array_equal(xf[:, 14], clear)
        lib.move(scenes.moved_placements(w, movable, 1))
        assert np.array_equal(lib.transforms()[:, 14], clear)
    finally:
        lib.close()
    orc = OracleScene.instanced(w.geometries, w.instances, movable)
    orc.set_clear(clear)
    ob, oo = orc.coverage()
    orc.close()
    assert np.array_equal(blas, ob)
    obj_cmp = obj.copy()
    obj_cmp[:, 13] = 0.0
    assert np.array_equal(obj_cmp, oo)


def test_prefiltered_sky_cones_cut_the_work_and_stay_close():
    f = scenes.icosphere_field(seed=5, n_spheres=12, subdivisions=4, width=48, height=27)
    o = OracleScene(f.meshes)
    exact = o.sky_visibility(f.receivers)
    pre = o.sky_visibility(f.receivers, prefilter=1.0)
    assert pre["work"][:, 2].mean() < 0.01 * exact["work"][:, 2].mean()
    assert np.abs(pre["irradiance"] - exact["irradiance"]).mean() < 1e-3 * math.pi
    # Light cones: prefilter 0 is the exact walk, bit for bit.
    a = o.visibility(f.receivers, f.lights)
    b = o.visibility(f.receivers, f.lights, prefilter=0.0)
    assert np.array_equal(a["fraction"], b["fraction"]) and np.array_equal(a["full"], b["full"])
