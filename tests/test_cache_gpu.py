"""The lighting cache's bake on a B200 (cc_cache_*): pages planned frame by
frame within the budget; every baked texel's pool value is the kernel's
result for that receiver (bit for bit), and within the parity bar of the
oracle's; texels without a surface hold 0 and texels past the grid nothing."""
import numpy as np
import pytest

import parity
from continuum_b200 import Light, LightingCache, RectLight, SphereLight, light_gpu, scenes
from oracle.oracle import SUM_FIXED, OracleScene

pytestmark = pytest.mark.gpu


def workload():
    w = scenes.box_field(grid=96)
    lights = np.stack([w.lights[0], light_gpu(Light(SphereLight((3.0, 5.0, -2.0), 0.6), (2.0, 1.5, 1.0)))])
    grid = w.receivers.reshape(96, 96, 8).copy()
    surface = np.ones((96, 96), bool)
    surface[::7, ::5] = False  # texels without a surface
    return w, lights, grid, surface


def bake_all(kernel, scene, lights, page_list, **opt):
    cache = LightingCache(kernel, scene, lights, **opt)
    frames = []
    for _ in range(200):
        st = cache.frame(page_list)
        frames.append(st)
        if st["pages_planned"] == 0 and st["resident"] == len(page_list):
            break
    return cache, frames


@pytest.mark.parametrize("light_ratio", [True, False])
def test_bake_matches_the_kernel_and_the_oracle(kernel, light_ratio):
    w, lights, grid, surface = workload()
    pages = scenes.grid_pages(grid, surface)
    for i, p in enumerate(pages):
        p.priority = (i * 7919) % 1000
    scene = kernel.scene(w.meshes)
    try:
        cache, frames = bake_all(kernel, scene, lights, pages, pages=4096, bake_budget=6000, light_ratio=light_ratio)
        assert frames[-1]["resident"] == len(pages)
        # The budget held each frame (a page costs 64 inside texels x 2 lights).
        assert all(f["spent"] <= 6000 for f in frames)
        assert sum(f["pages_planned"] for f in frames) == len(pages)
        # The direct path on the same receivers.
        rec = grid.reshape(-1, 8)
        got = kernel.visibility(scene, rec, lights, outputs=("irradiance", "fraction"))
        want = (got.fraction if light_ratio else got.irradiance).reshape(2, 96, 96)
        checked = 0
        for p in pages:
            vals = cache.read(p.key).reshape(9, 9, 2)
            _, py, px = p.key
            t = p.texels.reshape(9, 9, 8)
            for y in range(9):
                for x in range(9):
                    flag = t[y, x, 3]
                    if flag == 0.0:
                        assert np.all(vals[y, x] == 0.0)
                    elif flag == 1.0:
                        assert np.all(vals[y, x] == 0.0)
                    else:
                        assert np.array_equal(vals[y, x], want[:, py * 8 + y, px * 8 + x])
                        checked += 1
        assert checked > 0.9 * len(pages) * 64
        # And the oracle on the same receivers, within the parity bar.
        o = OracleScene(w.meshes).visibility(rec, lights, partial=False)
        d = np.abs(want.reshape(-1) - (o["fraction"] if light_ratio else o["irradiance"]))
        on = surface.reshape(-1)
        d = d.reshape(2, -1)[:, on]
        if light_ratio:
            assert d.max() <= parity.FRACTION_TOL
        else:
            u = o["unshadowed"].reshape(2, -1)[:, on]
            scale = np.maximum(u, parity.IRRADIANCE_FLOOR * u.max())
            assert (d / scale).max() <= parity.IRRADIANCE_TOL
        cache.close()
    finally:
        scene.close()


def test_adaptive_budget_uses_the_measured_bake_time(kernel):
    w, lights, grid, surface = workload()
    pages = scenes.grid_pages(grid, surface)
    scene = kernel.scene(w.meshes)
    try:
        cache = LightingCache(kernel, scene, lights, pages=4096, bake_budget=1 << 20, frame_target_ms=14.0)
        budgets, bake = [], []
        for f in range(12):
            st = cache.frame(pages, period_ms=16.0, render_ms=4.0)
            budgets.append(st["budget"])
            bake.append(st["last_bake_ms"])
        assert budgets[0] == 8000.0  # START_BUDGET
        assert bake[0] < 0 and all(b > 0 for b in bake[1:6])
        # The model steers the budget once timings arrive (odd frames 20 % lower).
        assert budgets[3] != budgets[2]
        jobs, slots = cache.jobs()
        assert jobs.shape[1] == 2
        cache.close()
    finally:
        scene.close()


def test_jobs_and_pool_layout(kernel):
    w, lights, grid, surface = workload()
    pages = scenes.grid_pages(grid[:24, :24], surface[:24, :24])
    scene = kernel.scene(w.meshes)
    try:
        cache = LightingCache(kernel, scene, lights, pages=64, bake_budget=1 << 20)
        st = cache.frame(pages)
        assert st["pages_planned"] == len(pages) == 9
        jobs, slots = cache.jobs()
        assert jobs.shape[0] == 9 * 81 * 2  # listed texels (inside 9 + 1, at most 9) x lights
        assert set(jobs[:, 1] >> 8) == {0, 1}
        ptr, ch = cache.pool()
        assert ptr != 0 and ch == 2
        with pytest.raises(Exception):
            cache.read((9, 9, 9))
        cache.close()
    finally:
        scene.close()


def terminator_workload():
    """A convex sphere (an undisplaced icosphere) lit from its side by a rect
    light, with a wall between the light and part of its far side, and a
    sphere light above; one texel per sphere triangle (its centroid lifted
    1e-4 along its normal, naming the triangle), laid out as a 40 x 32 grid."""
    sphere = scenes.displaced_icosphere((0.0, 0.0, 0.0), 1.0, seed=1, subdivisions=3, amplitude=0.0)
    wall = scenes.box_mesh((2.0, -3.0, 0.2), (2.2, 3.0, 3.0))
    tris = sphere.reshape(-1, 3, 3).astype(np.float64)
    n = np.cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    c = tris.mean(axis=1) + 1e-4 * n
    rec = np.zeros((len(tris), 8), np.float32)
    rec[:, 0:3], rec[:, 4:7] = c, n
    rec[:, 7] = (np.arange(len(tris), dtype=np.uint32) + 1).view(np.float32)  # own triangle + 1
    rect = light_gpu(Light.rect(RectLight((6.0, -0.5, -0.5), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), one_sided=False)))
    lights = np.stack([rect, light_gpu(Light(SphereLight((0.3, 6.0, 0.2), 0.5), (1.0, 1.0, 1.0)))])
    return [sphere, wall], np.ascontiguousarray(rec[:1280]), lights


@pytest.mark.parametrize("light_ratio", [True, False])
def test_back_facing_texels_bake_the_share_past_their_own_triangle(kernel, light_ratio):
    """vc_bake's `back` (mask_cones.wgsl:3476-3494): a light below a texel's
    horizon bakes the share seen past the texel's own triangle (1 on the
    convex sphere's terminator, less where the wall covers the light) and no
    light; the pool equals cc_visibility with CC_BACK_FACING bit for bit and
    the oracle's estimator within the parity bar."""
    from continuum_b200 import _lib

    meshes, rec, lights = terminator_workload()
    grid = rec.reshape(40, 32, 8)
    pages = scenes.grid_pages(grid)
    scene = kernel.scene(meshes)
    try:
        cache, frames = bake_all(kernel, scene, lights, pages, pages=256, bake_budget=1 << 16, light_ratio=light_ratio)
        got = kernel.visibility(scene, rec, lights, outputs=("irradiance", "fraction", "full", "any"),
                                flags=_lib.CC_BACK_FACING)
        want = (got.fraction if light_ratio else got.irradiance).reshape(2, 40, 32)
        for p in pages:
            vals = cache.read(p.key).reshape(9, 9, 2)
            _, py, px = p.key
            for y in range(min(9, 40 - py * 8)):
                for x in range(min(9, 32 - px * 8)):
                    assert np.array_equal(vals[y, x], want[:, py * 8 + y, px * 8 + x]), (p.key, y, x)
        cache.close()
        o = OracleScene(meshes)
        orc = o.visibility(rec, lights, back_facing=True, accumulate=SUM_FIXED)
        g = {"full": got.full.reshape(-1), "any": got.any.reshape(-1), "fraction": got.fraction.reshape(-1),
             "irradiance": got.irradiance.reshape(-1)}
        parity.compare(g, orc, orc["unshadowed"])
        plain = kernel.visibility(scene, rec, lights, outputs=("fraction",))
        open_light = o.visibility(rec, lights, partial=False)["unshadowed"].reshape(2, -1)[0]
        o.close()
    finally:
        scene.close()
    # Texels below the rect light's horizon: without the estimator their
    # ratio is 1; with it, 1 where only their own sphere turns away, less
    # where the wall covers the light, and their light is 0.
    below = open_light <= 0.0
    frac = got.fraction.reshape(2, -1)[0]
    assert below.sum() > 500
    assert np.all(plain.fraction.reshape(2, -1)[0][below] == 1.0)
    assert np.all(got.irradiance.reshape(2, -1)[0][below] == 0.0)
    assert (frac[below] == 1.0).mean() > 0.3 and (frac[below] < 0.9).sum() > 100  # the wall's shadow
    # The sphere alone: every texel below the light's horizon sees all of it
    # past its own triangle (a convex object's terminator).
    alone = kernel.scene(meshes[:1])
    try:
        v = kernel.visibility(alone, rec, lights, outputs=("fraction",), flags=_lib.CC_BACK_FACING)
    finally:
        alone.close()
    assert np.all(v.fraction.reshape(2, -1)[0][below] == 1.0)
