"""Parity of the CUDA path with the oracle, through the C ABI, on a B200.

Every case runs the library (include/continuum_cuda.h via ctypes) and the
oracle on the same seeded inputs and holds them to the bar in tests/parity.py.
"""
import numpy as np
import pytest

import kat
import parity
from continuum_b200 import Hierarchy, Light, RectLight, SphereLight, Spot, _lib, light_gpu, scenes
from oracle.oracle import OracleScene

pytestmark = pytest.mark.gpu

ALL = ("full", "any", "partial", "irradiance", "fraction", "work")


def run_both(kernel, meshes, rec, lights, hierarchy=2, ppw=None, **caps):
    scene = kernel.scene(meshes)
    for k, v in caps.items():
        setattr(kernel, k, v)
    try:
        g = kernel.visibility(scene, rec, lights, hierarchy=hierarchy, outputs=ALL, points_per_warp=ppw)
    finally:
        kernel.wide_extent, kernel.light_cone_cap, kernel.wide_cone_cap = 8.0, 4096, 512
        scene.close()
    o = OracleScene(meshes).visibility(rec, lights, hierarchy=hierarchy, **caps)
    return parity.flat(g), o


@pytest.mark.parametrize("hierarchy", [0, 1, 2])
def test_box_field(kernel, hierarchy):
    """The small plain workload (65,536 cones), every hierarchy mode."""
    w = scenes.box_field()
    g, o = run_both(kernel, w.meshes, w.receivers, w.lights, hierarchy)
    stats = parity.compare(g, o, o["unshadowed"])
    assert stats["cones"] == 65536


def test_cones_match_the_cpu(kernel):
    """The reference's GPU test (gpu.rs:294-337) through irradiance()."""
    meshes = kat.four_boxes()
    rec = kat.grid_floor(48)
    gpu, secs = kernel.irradiance(rec[:, [0, 1, 2, 4, 5, 6]], kat.CEILING, meshes, runs=2)
    cpu, total = OracleScene(meshes).cpu_masked(rec, kat.light9(kat.CEILING))
    worst = float(np.max(np.abs(cpu - gpu) / total))
    assert worst <= 1e-4, worst
    assert secs > 0.0


def test_m2_gate1_room(kernel):
    """M2 gate 1: 256 x 256 receivers in the gate 1 room within 1e-4 of the
    light's weight of the CPU path, through irradiance() and irradiance_with()."""
    meshes = kat.gate1_room()
    rec = kat.floor_points(256)
    r6 = rec[:, [0, 1, 2, 4, 5, 6]]
    cpu, total = OracleScene(meshes).cpu_masked(rec, kat.light9(kat.CEILING))
    for h in (Hierarchy.NONE, True, Hierarchy.MESHES):
        gpu, _ = kernel.irradiance_with(r6, kat.CEILING, meshes, h)
        assert float(np.max(np.abs(cpu - gpu) / total)) <= 1e-4


def test_a_large_wall_shadows_receivers_close_to_it(kernel):
    """gpu.rs:362-393 through irradiance()."""
    light = kat.sun_behind_the_wall()
    rec = kat.wall_receivers()[:, [0, 1, 2, 4, 5, 6]]
    open_, _ = kernel.irradiance(rec, light, [])
    shadowed, _ = kernel.irradiance(rec, light, kat.wall())
    assert np.all(open_ > 0.0)
    assert float(np.max(shadowed / np.maximum(open_, 1e-12))) <= 5e-3


def test_coverage_matches_the_oracle(kernel):
    """coverage() (lib.rs:3289-3298): 64 per-bin coverages per receiver."""
    meshes = kat.four_boxes()
    rec = kat.grid_floor(32)
    cov = kernel.coverage(rec[:, [0, 1, 2, 4, 5, 6]], kat.CEILING, meshes)
    o = OracleScene(meshes).visibility(rec, kat.lights16(kat.CEILING), hierarchy=0)
    assert cov.shape == (1024, 64)
    assert float(np.max(np.abs(cov - o["partial"]))) <= 1e-4


def test_packets_equal_solo_walks(kernel):
    """Packet traversal changes no result (the reference's packet_check): one
    cone per warp and 32 per warp give identical bits and values."""
    w = scenes.box_field(grid=128)
    scene = kernel.scene(w.meshes)
    runs = [parity.flat(kernel.visibility(scene, w.receivers, w.lights, outputs=ALL, points_per_warp=p))
            for p in (1, 8, 32)]
    scene.close()
    for r in runs[1:]:
        for k in ("full", "any", "partial", "irradiance", "fraction"):
            assert np.array_equal(r[k], runs[0][k]), k


def test_walk_order_changes_no_result(kernel):
    """Walking points in Morton order (the default) or in the given order
    (CC_KEEP_ORDER) gives identical results."""
    w = small_field(seed=11, n=8, sub=3, width=96, height=54)
    scene = kernel.scene(w.meshes)
    a = parity.flat(kernel.visibility(scene, w.receivers, w.lights, outputs=ALL))
    b = parity.flat(kernel.visibility(scene, w.receivers, w.lights, outputs=ALL, flags=_lib.CC_KEEP_ORDER))
    scene.close()
    for k in ("full", "any", "partial", "irradiance", "fraction"):
        assert np.array_equal(a[k], b[k]), k


def test_split_chunks_change_no_result(kernel):
    """Exact cones are set up, walked and integrated a chunk at a time; chunks
    of any size (whole packets or not) give identical results."""
    w = small_field(seed=13, n=8, sub=3, width=96, height=54)
    scene = kernel.scene(w.meshes)
    base = parity.flat(kernel.visibility(scene, w.receivers, w.lights, outputs=ALL))
    try:
        for chunk in (32, 1000, 4099):
            kernel.set_split_chunk(chunk)
            got = parity.flat(kernel.visibility(scene, w.receivers, w.lights, outputs=ALL))
            for k in ("full", "any", "partial", "irradiance", "fraction"):
                assert np.array_equal(got[k], base[k]), (chunk, k)
        with pytest.raises(_lib.CCError):
            kernel.set_split_chunk(31)
    finally:
        kernel.set_split_chunk(1 << 25)
        scene.close()


def test_host_buffers_with_full_and_any_only(kernel):
    """Host-buffer calls download FULL and ANY on a second stream while the
    integration runs; asked for alone (no irradiance or fraction), over one
    chunk or several, they equal the words of a call that asks for all."""
    w = small_field(seed=17, n=8, sub=3, width=96, height=54)
    scene = kernel.scene(w.meshes)
    base = kernel.visibility(scene, w.receivers, w.lights, outputs=ALL)
    try:
        for chunk in (1 << 25, 1000):
            kernel.set_split_chunk(chunk)
            got = kernel.visibility(scene, w.receivers, w.lights, outputs=("full", "any"))
            assert np.array_equal(got.full, base.full), chunk
            assert np.array_equal(got.any, base.any), chunk
            assert not hasattr(got, "irradiance") or got.irradiance is None
    finally:
        kernel.set_split_chunk(1 << 25)
        scene.close()


def small_field(seed=5, n=12, sub=4, width=160, height=90):
    return scenes.icosphere_field(seed=seed, n_spheres=n, subdivisions=sub, width=width, height=height)


def test_icosphere_field_small(kernel):
    """A scaled-down plain-at-scale workload: displaced icospheres, two rect
    and two sphere (disk) lights with spots, camera primary hits."""
    w = small_field()
    g, o = run_both(kernel, w.meshes, w.receivers, w.lights)
    stats = parity.compare(g, o, o["unshadowed"])
    assert stats["cones"] == 4 * 160 * 90


def test_walk_caps_and_solo_rewalks(kernel):
    """Low walk caps make many walks stop early; the cut depends on the walk
    order, so the packets' order-diverged cones are walked again alone and
    every result equals the oracle's own solo walk."""
    w = small_field(seed=7, n=20, sub=4)
    g, o = run_both(kernel, w.meshes, w.receivers, w.lights, light_cone_cap=48, wide_cone_cap=16)
    capped = (g["work"][:, 3] & _lib.CC_CONE_CAPPED) != 0
    assert capped.mean() > 0.01
    parity.compare(g, o, o["unshadowed"])


def test_wide_and_grazing_cones(kernel):
    """Receivers near a large light's plane (wide windows, clipped or grazing)
    and near a sphere light (a clipped sphere window)."""
    big = RectLight((-3.0, 0.3, -3.0), (6.0, 0.0, 0.0), (0.0, 0.0, 6.0), one_sided=False)
    sphere = Light(SphereLight((0.0, 0.6, 0.0), 0.5))
    xs = np.linspace(-6, 6, 64, dtype=np.float32)
    pts = np.stack(np.meshgrid(xs, [0.05, 0.29], xs, indexing="ij"), -1).reshape(-1, 3)
    rec = kat.receivers(pts, (0.0, 1.0, 0.0))
    meshes = [scenes.box_mesh((x, 0.1, z), (x + 0.3, 0.2, z + 0.3)) for x in range(-5, 5, 2) for z in range(-5, 5, 2)]
    lights = np.stack([light_gpu(Light.rect(big)), light_gpu(sphere)])
    g, o = run_both(kernel, meshes, rec, lights)
    parity.compare(g, o, o["unshadowed"])


def test_flat_scene_upload_equals_build(kernel):
    """A scene uploaded from the reference's flattened arrays (as the oracle
    builds them) gives the same results as the library's own build."""
    w = small_field(seed=9, n=6, sub=3, width=64, height=36)
    os_ = OracleScene(w.meshes)
    a = os_.arrays()
    tris12 = np.zeros((os_.tri9.shape[0], 12), np.float32)
    tris12[:, [0, 1, 2, 4, 5, 6, 8, 9, 10]] = os_.tri9
    s1 = kernel.scene_from_flat(tris12, a["ranges"], a["blas"], a["blas_items"], a["nodes"], a["items"])
    s2 = kernel.scene(w.meshes)
    r1 = parity.flat(kernel.visibility(s1, w.receivers, w.lights, outputs=ALL))
    r2 = parity.flat(kernel.visibility(s2, w.receivers, w.lights, outputs=ALL))
    for k in ("full", "any", "partial", "irradiance", "fraction"):
        assert np.array_equal(r1[k], r2[k]), k


def test_invalid_flat_scene_is_rejected(kernel):
    w = small_field(seed=9, n=2, sub=1, width=8, height=8)
    a = OracleScene(w.meshes).arrays()
    nodes = a["nodes"].copy()
    nodes[0]["info"][0] = 10_000  # child beyond the array
    tris12 = np.zeros((w.ntris, 12), np.float32)
    with pytest.raises(_lib.CCError) as e:
        kernel.scene_from_flat(tris12, a["ranges"], a["blas"], a["blas_items"], nodes, a["items"])
    assert e.value.code == _lib.CC_ERR_INVALID


def test_edge_cases(kernel):
    """No meshes, an empty mesh among others, a degenerate triangle,
    receivers facing away, behind a one-sided light, and in the light's plane."""
    light = RectLight((-0.5, 2.0, -0.5), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0), one_sided=True)  # faces down
    pts = [(0, 0, 0), (0.2, 0.0, 0.1), (0, 3.0, 0), (0, 2.0, 0), (3, 0, 3), (0.1, 0.0, -0.2)]
    nrm = np.array([(0, 1, 0), (0, -1, 0), (0, 1, 0), (0, 1, 0), (0, 1, 0), (0, 1, 0)], np.float32)
    rec = kat.receivers(pts, (0, 1, 0))
    rec[:, 4:7] = nrm
    degenerate = np.array([[[0, 1, 0], [1, 1, 0], [2, 1, 0]]], np.float32)
    for meshes in ([], [np.zeros((0, 3, 3), np.float32), scenes.box_mesh((-0.2, 0.5, -0.2), (0.2, 0.6, 0.2)),
                        degenerate]):
        g, o = run_both(kernel, meshes, rec, kat.lights16(light))
        parity.compare(g, o, o["unshadowed"])
    # Zero receivers and zero lights are no work, not errors.
    scene = kernel.scene([scenes.box_mesh((0, 0, 0), (1, 1, 1))])
    v = kernel.visibility(scene, np.zeros((0, 8), np.float32), kat.lights16(light))
    assert v.fraction.shape == (1, 0)
    scene.close()


def test_device_pointers_and_streams(kernel):
    """Inputs and outputs resident on the device, on a torch stream, give the
    host path's results."""
    import torch

    w = scenes.box_field(grid=64)
    scene = kernel.scene(w.meshes)
    host = parity.flat(kernel.visibility(scene, w.receivers, w.lights, outputs=ALL))
    dev = torch.device("cuda:0")
    rec = torch.from_numpy(w.receivers).to(dev)
    lig = torch.from_numpy(w.lights).to(dev)
    n = rec.shape[0] * lig.shape[0]
    outs = {"full": torch.zeros(n, dtype=torch.int64, device=dev), "any": torch.zeros(n, dtype=torch.int64, device=dev),
            "partial": torch.zeros(n, 64, device=dev), "irradiance": torch.zeros(n, device=dev),
            "fraction": torch.zeros(n, device=dev)}
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        kernel.visibility_device(scene, rec.data_ptr(), rec.shape[0], lig.data_ptr(), lig.shape[0],
                                 {k: v.data_ptr() for k, v in outs.items()}, stream=stream.cuda_stream)
    stream.synchronize()
    assert np.array_equal(outs["full"].cpu().numpy().view(np.uint64), host["full"])
    assert np.array_equal(outs["any"].cpu().numpy().view(np.uint64), host["any"])
    assert np.array_equal(outs["fraction"].cpu().numpy(), host["fraction"])
    assert np.array_equal(outs["partial"].cpu().numpy(), host["partial"])
    scene.close()


def test_golden_fixtures(kernel):
    """The committed fixtures (tests/golden, made by the oracle) still hold."""
    from golden_fixtures import check_all

    check_all(kernel)


def test_stacked_layers_overflow_to_wide_accumulators(kernel):
    """One mesh of 200 stacked quads over the receivers piles 200 bins' worth
    of coverage into each cell: the packet pass's 32-bit accumulators
    overflow, the cones are walked again with 64-bit ones (status
    CC_CONE_ACC_WIDE), and the results are the oracle's."""
    quads = []
    for k in range(200):
        y = 1.0 + 0.01 * k
        # Wound to face the receivers below (a triangle facing away is culled).
        quads.append(np.array([[[-2, y, -2], [2, y, 2], [-2, y, 2]], [[-2, y, -2], [2, y, -2], [2, y, 2]]],
                              np.float32))
    stack = np.concatenate(quads)
    light = RectLight((-0.5, 4.0, -0.5), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0))
    xs = np.linspace(-1.0, 1.0, 16, dtype=np.float32)
    pts = np.stack(np.meshgrid(xs, [0.0], xs, indexing="ij"), -1).reshape(-1, 3)
    rec = kat.receivers(pts, (0.0, 1.0, 0.0))
    g, o = run_both(kernel, [stack], rec, kat.lights16(light))
    wide = (g["work"][:, 3] & _lib.CC_CONE_ACC_WIDE) != 0
    assert wide.mean() > 0.5
    parity.compare(g, o, o["unshadowed"])
    assert np.all(g["full"] == np.uint64(0xFFFFFFFFFFFFFFFF))
