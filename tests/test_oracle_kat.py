"""The oracle pinned against the reference's own known-answer tests.

The oracle restates the reference's WGSL light-cone path (the GPU semantics
the CUDA library must match). Here it is checked, on the CPU, against every
test the reference holds for this path, with the reference's tolerances:
its GPU-vs-CPU test, its large-wall test, the cone3 unit tests, the BVH
candidates test, the M2 gate 1 room and the hierarchy-equals-brute-force
check. The reference's CPU path (cone3 + coverage + bvh) is restated in the
oracle too and serves as the second side of those comparisons.
"""
import numpy as np
import pytest

import kat
from oracle.oracle import OracleScene, cpu_weights, disk_table, poly_overflows


def _wgsl_visible(meshes, rec, rect, hierarchy=0):
    s = OracleScene(meshes)
    r = s.visibility(rec, kat.lights16(rect), hierarchy=hierarchy)
    s.close()
    return r


def test_cones_match_the_cpu():
    """gpu.rs:294-337: the GPU path within 1e-4 of the light's weight of the
    CPU path at every receiver (48 x 48, four boxes)."""
    meshes = kat.four_boxes()
    rec = kat.grid_floor(48)
    r = _wgsl_visible(meshes, rec, kat.CEILING, hierarchy=0)
    s = OracleScene(meshes)
    cpu, total = s.cpu_masked(rec, kat.light9(kat.CEILING))
    worst = float(np.max(np.abs(cpu - r["irradiance"]) / total))
    assert worst <= 1e-4, worst
    # The same with both hierarchy levels (irradiance_with(.., true, ..)).
    r2 = _wgsl_visible(meshes, rec, kat.CEILING, hierarchy=2)
    assert float(np.max(np.abs(cpu - r2["irradiance"]) / total)) <= 1e-4


def test_m2_gate1_room_matches_the_cpu():
    """M2 gate 1 (experiments/room3d/src/bin/m2_gate1.rs, docs/results/m2-gate1.md):
    256 x 256 floor receivers in the gate 1 room, every receiver within 1e-4 of
    the light's weight (the reference recorded 6.4e-6 on an M4)."""
    meshes = kat.gate1_room()
    rec = kat.floor_points(256)
    r = _wgsl_visible(meshes, rec, kat.CEILING, hierarchy=0)
    s = OracleScene(meshes)
    cpu, total = s.cpu_masked(rec, kat.light9(kat.CEILING))
    diff = np.abs(cpu - r["irradiance"]) / total
    assert float(diff.max()) <= 1e-4, float(diff.max())
    assert int((diff > 1e-4).sum()) == 0


def test_a_large_wall_shadows_receivers_close_to_it():
    """gpu.rs:362-393: no receiver sees more than 0.5% of its unshadowed light."""
    light = kat.sun_behind_the_wall()
    rec = kat.wall_receivers()
    s_open = OracleScene([])
    open_ = s_open.visibility(rec, kat.lights16(light), hierarchy=0)["irradiance"]
    shadowed = _wgsl_visible(kat.wall(), rec, light, hierarchy=0)["irradiance"]
    assert np.all(open_ > 0.0)
    worst = float(np.max(shadowed / np.maximum(open_, 1e-12)))
    assert worst <= 5e-3, worst


@pytest.mark.parametrize("p", [(0.5, 0.5, 0.0), (0.1, 0.8, 0.0), (0.9, 0.3, 0.2)])
def test_bin_weights_sum_to_the_lights_projected_solid_angle(p):
    """cone3.rs:539-554: bin weights vs 256^2 stratified samples, 1e-3 relative
    (CPU cone weights, and the WGSL path's open irradiance)."""
    reference = kat.sampled_visible(p, [], 256)
    w = cpu_weights(p, (0, 0, 1), kat.light9(kat.CEILING))
    assert abs(float(w.sum()) - reference) / reference < 1e-3
    rec = kat.receivers([p], (0.0, 0.0, 1.0))
    irr = _wgsl_visible([], rec, kat.CEILING)["irradiance"][0]
    assert abs(float(irr) - reference) / reference < 1e-3


def test_a_box_blocking_everything_leaves_nothing():
    """cone3.rs:556-566."""
    rec = kat.receivers([(0.5, 0.5, 0.0)], (0.0, 0.0, 1.0))
    meshes = [kat.box_mesh((0.2, 0.2, 0.4), (0.8, 0.8, 0.5))]
    r = _wgsl_visible(meshes, rec, kat.CEILING)
    assert float(r["irradiance"][0]) < 1e-6
    assert r["full"][0] == np.uint64(0xFFFFFFFFFFFFFFFF)
    assert float(r["fraction"][0]) == 0.0
    cpu, _ = OracleScene(meshes).cpu_masked(rec, kat.light9(kat.CEILING))
    assert float(cpu[0]) < 1e-6


def test_mask_cone_matches_sampled_visibility():
    """cone3.rs:568-590: within 0.02 of the cone's weight of 128^2 sampled rays."""
    meshes = [kat.box_mesh((0.35, 0.3, 0.4), (0.5, 0.7, 0.45)), kat.box_mesh((0.55, 0.45, 0.6), (0.62, 0.52, 0.7))]
    for p in [(0.5, 0.5, 0.0), (0.42, 0.55, 0.0), (0.7, 0.4, 0.0)]:
        rec = kat.receivers([p], (0.0, 0.0, 1.0))
        masked = float(_wgsl_visible(meshes, rec, kat.CEILING)["irradiance"][0])
        reference = kat.sampled_visible(p, meshes, 128)
        total = float(cpu_weights(p, (0, 0, 1), kat.light9(kat.CEILING)).sum())
        assert abs(masked - reference) < 0.02 * total, (p, masked, reference)


def test_internal_mesh_edges_do_not_leak():
    """cone3.rs:592-611: a box covering half the window blocks exactly its half."""
    p = (0.5, 0.5, 0.0)
    rec = kat.receivers([p], (0.0, 0.0, 1.0))
    meshes = [kat.box_mesh((0.0, 0.0, 0.5), (0.5, 1.0, 0.55))]
    w = cpu_weights(p, (0, 0, 1), kat.light9(kat.CEILING))
    left_half = float(sum(w[b] for b in range(64) if b % 8 < 4))
    total = float(w.sum())
    vis = float(_wgsl_visible(meshes, rec, kat.CEILING)["irradiance"][0])
    assert abs(vis - (total - left_half)) < 1e-4 * total
    cpu, _ = OracleScene(meshes).cpu_masked(rec, kat.light9(kat.CEILING))
    assert abs(float(cpu[0]) - (total - left_half)) < 1e-4 * total


def test_geometry_beyond_the_light_does_not_occlude():
    """cone3.rs:613-623."""
    p = (0.5, 0.5, 0.0)
    rec = kat.receivers([p], (0.0, 0.0, 1.0))
    meshes = [kat.box_mesh((0.2, 0.2, 1.1), (0.8, 0.8, 1.2))]
    total = float(cpu_weights(p, (0, 0, 1), kat.light9(kat.CEILING)).sum())
    r = _wgsl_visible(meshes, rec, kat.CEILING)
    assert abs(float(r["irradiance"][0]) - total) < 1e-6
    assert r["any"][0] == 0 and float(r["fraction"][0]) == 1.0


def test_bvh_candidates_match_brute_force():
    """bvh.rs:173-214 and M1 gate 2 (hierarchy = brute force within 2.5e-6):
    the CPU path with its leaf-4 BVH equals brute-force culling, and the WGSL
    path's hierarchies equal testing every triangle."""
    meshes = [kat.box_mesh((0.05 * i, 0.3, 0.4 + 0.01 * i), (0.05 * i + 0.03, 0.7, 0.42 + 0.01 * i))
              for i in range(20)]
    meshes.append(kat.sphere_mesh((0.5, 0.5, 0.6), 0.1, 24, 12))
    rec = kat.receivers([(0.5, 0.5, 0.0), (0.1, 0.9, 0.0), (0.8, 0.2, 0.0)], (0.0, 0.0, 1.0))
    s = OracleScene(meshes)
    brute, total = s.cpu_masked(rec, kat.light9(kat.CEILING), use_bvh=False)
    bvh, _ = s.cpu_masked(rec, kat.light9(kat.CEILING), use_bvh=True)
    assert np.all(np.abs(brute - bvh) <= 2.5e-6 * total)
    lig = kat.lights16(kat.CEILING)
    r0 = s.visibility(rec, lig, hierarchy=0)
    for h in (1, 2):
        rh = s.visibility(rec, lig, hierarchy=h)
        assert np.array_equal(r0["full"], rh["full"]) and np.array_equal(r0["any"], rh["any"])
        assert np.all(np.abs(r0["irradiance"] - rh["irradiance"]) <= 2.5e-6 * total)


def test_rubble_room_hierarchy_equals_brute_force():
    """M1 gate 2's scene with 3,000 boxes (room3d with_rubble): the hierarchy
    walk and testing every triangle agree within 2.5e-6 of the light's weight."""
    meshes = kat.with_rubble()
    rec = kat.floor_points(64)
    s = OracleScene(meshes)
    lig = kat.lights16(kat.CEILING)
    r0 = s.visibility(rec, lig, hierarchy=0, partial=False)
    r2 = s.visibility(rec, lig, hierarchy=2, partial=False)
    _, total = s.cpu_masked(rec, kat.light9(kat.CEILING))
    assert np.all(np.abs(r0["irradiance"] - r2["irradiance"]) <= 2.5e-6 * total)
    assert np.mean(r0["full"] == r2["full"]) >= 0.999


def test_disk_table_is_the_references():
    """The sphere light's inscribed-disk bin fractions (mask_cones.wgsl:888-897),
    computed from geometry, equal the reference's six-decimal table."""
    t = disk_table().reshape(8, 8)
    # The reference's first two rows (a golden vector); the rest follows by symmetry.
    row0 = [0.000000, 0.160355, 0.694958, 0.957934, 0.957934, 0.694958, 0.160355, 0.000000]
    row1 = [0.160355, 0.939877, 1.0, 1.0, 1.0, 1.0, 0.939877, 0.160355]
    assert np.allclose(t[0], row0, atol=1e-9) and np.allclose(t[1], row1, atol=1e-9)
    assert np.allclose(t, t[::-1]) and np.allclose(t, t[:, ::-1]) and np.allclose(t, t.T)
    assert np.allclose(t[2:6, 1:7], 1.0)


def test_fp64_and_fp32_oracles_agree():
    """The FP64 restatement stays within the path's tolerances of the FP32 one."""
    from continuum_b200 import scenes

    w = scenes.box_field(grid=64)
    s = OracleScene(w.meshes)
    r32 = s.visibility(w.receivers, w.lights, precision=4)
    r64 = s.visibility(w.receivers, w.lights, precision=8)
    assert np.max(np.abs(r32["fraction"] - r64["fraction"])) <= 1e-3
    assert np.mean(r32["full"] == r64["full"]) >= 0.999
    assert poly_overflows() == 0


def test_oracle_reproduces_the_golden_fixtures():
    """The oracle still gives the committed fixtures' values (within the bar)."""
    import golden_fixtures
    from oracle.oracle import OracleScene
    import parity

    for name, (meshes, rec, lights, h, _) in golden_fixtures.cases().items():
        r = OracleScene(meshes).visibility(rec, lights, hierarchy=h)
        stats = golden_fixtures.check(name, r)
        assert stats["word_agreement"] == 1.0
    for name, (w, clear, pf, _) in golden_fixtures.instanced_cases().items():
        stats = golden_fixtures.check(name, golden_fixtures.oracle_instanced(w, clear, pf))
        assert stats["word_agreement"] == 1.0
