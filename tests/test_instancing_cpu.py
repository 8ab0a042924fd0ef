"""Instanced scenes on the CPU: the library's host builder lays out objects,
transforms and hierarchies exactly as the oracle's restatement of
flatten_instanced and object_hierarchy does, and the camera pass casts rays
into each object's space."""
import numpy as np
import pytest

from continuum_b200 import _lib, host_scene_instanced, scenes
from oracle.oracle import OracleScene


def small_world(seed=3, n=300):
    return scenes.instanced_world(seed=seed, n_instances=n, n_boulders=3, half=40.0, n_lights=4, width=96,
                                  height=54, segments=24, rings=13)


def test_instanced_builder_matches_the_oracle():
    w = small_world()
    lib = host_scene_instanced(w.geometries, w.instances)
    orc = OracleScene.instanced(w.geometries, w.instances)
    a, b = lib.arrays(), orc.arrays()
    for k in ("ranges", "blas_items", "items"):
        assert np.array_equal(a[k], b[k]), k
    for k in ("blas", "nodes"):
        assert a[k].tobytes() == b[k].tobytes(), k
    assert np.array_equal(lib.transforms(), orc.transforms())
    ranges = a["ranges"]
    assert ranges.shape[0] == len(w.instances)
    assert np.array_equal(ranges[:, 3], np.arange(len(w.instances)))
    lib.close()
    orc.close()


def test_transforms_are_the_reference_rows():
    w = small_world(n=10)
    x = host_scene_instanced(w.geometries, w.instances).transforms()
    inst = w.instances
    rot = inst["rotation"].reshape(-1, 3, 3)
    assert np.array_equal(x[:, [0, 1, 2]], rot[:, 0])
    assert np.array_equal(x[:, [4, 5, 6]], rot[:, 1])
    assert np.array_equal(x[:, [8, 9, 10]], rot[:, 2])
    assert np.array_equal(x[:, [3, 7, 11]], inst["translation"])
    assert np.array_equal(x[:, 12], inst["scale"])
    assert np.array_equal(x[:, 13], (np.float32(1) / inst["scale"]).astype(np.float32))


def test_primary_hits_lie_on_placed_objects():
    """A boulder placed by a transform is hit where its world-space copy is."""
    w = small_world(n=40)
    hs = host_scene_instanced(w.geometries, w.instances)
    rec, hit = hs.primary_hits(w.camera, 96, 54)
    hs.close()
    # The same objects flattened to world space.
    meshes = []
    for o in w.instances:
        g = w.geometries[o["geometry"]].reshape(-1, 3).astype(np.float64)
        R = o["rotation"].reshape(3, 3).astype(np.float64)
        meshes.append(((g @ R.T) * float(o["scale"]) + o["translation"]).reshape(-1, 3, 3).astype(np.float32))
    from continuum_b200 import host_scene
    ws = host_scene(meshes)
    rec2, hit2 = ws.primary_hits(w.camera, 96, 54)
    ws.close()
    both = hit.astype(bool) & hit2.astype(bool)
    assert both.mean() > 0.9 * hit2.astype(bool).mean()
    np.testing.assert_allclose(rec[both, :3], rec2[both, :3], atol=2e-3)
    np.testing.assert_allclose(rec[both, 4:7], rec2[both, 4:7], atol=2e-3)


def test_invalid_instances_are_rejected():
    g = [scenes.box_mesh((0, 0, 0), (1, 1, 1))]
    bad_rot = np.zeros(1, _lib.INSTANCE_DTYPE)
    bad_rot[0] = (0, np.full(9, 0.5, np.float32), 1.0, (0, 0, 0))
    bad_geo = np.zeros(1, _lib.INSTANCE_DTYPE)
    bad_geo[0] = (3, np.eye(3, dtype=np.float32).reshape(9), 1.0, (0, 0, 0))
    bad_scale = np.zeros(1, _lib.INSTANCE_DTYPE)
    bad_scale[0] = (0, np.eye(3, dtype=np.float32).reshape(9), 0.0, (0, 0, 0))
    for inst in (bad_rot, bad_geo, bad_scale):
        with pytest.raises(_lib.CCError) as e:
            host_scene_instanced(g, inst)
        assert e.value.code == _lib.CC_ERR_INVALID


def test_movers_subtree_matches_the_oracle_before_and_after_a_move():
    w = small_world(n=300)
    movable = np.arange(0, 300, 10, dtype=np.uint32)
    lib = host_scene_instanced(w.geometries, w.instances, movable)
    orc = OracleScene.instanced(w.geometries, w.instances, movable)

    def same():
        a, b = lib.arrays(), orc.arrays()
        for k in ("ranges", "blas_items", "items"):
            assert np.array_equal(a[k], b[k]), k
        for k in ("blas", "nodes"):
            assert a[k].tobytes() == b[k].tobytes(), k
        assert np.array_equal(lib.transforms(), orc.transforms())
        return a

    a = same()
    assert a["nodes"][0]["info"][0] == 1 and a["nodes"][0]["info"][2] == 1  # root over the two subtrees
    for frame in (1, 2):
        pl = scenes.moved_placements(w, movable, frame)
        ba, bb = lib.move(pl), orc.move(pl)
        assert np.array_equal(ba, bb)
        a = same()
        # The movers' new bounds are inside the root's.
        assert np.all(ba[:, 6:9] >= a["nodes"][0]["lo"][:3]) and np.all(ba[:, 9:12] <= a["nodes"][0]["hi"][:3])
    lib.close()
    orc.close()


def test_moving_without_movers_is_an_error():
    w = small_world(n=20)
    s = host_scene_instanced(w.geometries, w.instances)
    with pytest.raises(_lib.CCError):
        s.move(w.instances[:1])
    s.close()
