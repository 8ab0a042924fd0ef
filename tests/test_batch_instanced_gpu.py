"""Instanced scenes in the batched and served forms, and batched update jobs
(cc_batch_add_update), on a B200: every result equals the plain call's for
the same job alone (cc_visibility, cc_visibility_update), bit for bit, on
the first (direct) submission and on graph replays."""
import numpy as np
import pytest

from continuum_b200 import Batch, Server, _lib, scenes

pytestmark = pytest.mark.gpu

KEYS = ("full", "any", "irradiance", "fraction")


@pytest.fixture(scope="module")
def world():
    return scenes.instanced_world(seed=3, n_instances=300, n_boulders=3, half=40.0, n_lights=4, width=96, height=54,
                                  segments=24, rings=13)


def outputs(torch, n, with_all=False):
    dev = torch.device("cuda:0")
    o = {"full": torch.zeros(n, dtype=torch.int64, device=dev), "any": torch.zeros(n, dtype=torch.int64, device=dev),
         "irradiance": torch.zeros(n, device=dev), "fraction": torch.zeros(n, device=dev)}
    if with_all:
        o["partial"] = torch.zeros(n, 64, device=dev)
        o["work"] = torch.zeros(n, 4, dtype=torch.int32, device=dev)
    return o


def ptrs(outs):
    return {k: v.data_ptr() for k, v in outs.items()}


def same(a, b, keys):
    for k in keys:
        assert np.array_equal(a[k].cpu().numpy(), b[k].cpu().numpy()), k


def test_instanced_and_world_space_jobs_share_a_batch(kernel, world):
    """An instanced job (two hierarchy levels and the flat object level) beside
    a world-space job: the batch runs the instanced kernel for all of them."""
    import torch

    inst = kernel.scene_instanced(world.geometries, world.instances)
    ico = scenes.icosphere_field(seed=8, n_spheres=6, subdivisions=3, width=64, height=36)
    flat = kernel.scene(ico.meshes)
    specs = [(inst, world.receivers, world.lights, 2), (flat, ico.receivers, ico.lights, 2),
             (inst, world.receivers[::5], world.lights[1:3], 1)]
    jobs = []
    for scene, rec, lig, h in specs:
        r = torch.from_numpy(np.ascontiguousarray(rec)).cuda()
        l = torch.from_numpy(np.ascontiguousarray(lig)).cuda()
        jobs.append((scene, r, l, h, outputs(torch, r.shape[0] * l.shape[0], with_all=True)))
    alone = []
    for scene, r, l, h, outs in jobs:
        ref = {k: torch.zeros_like(v) for k, v in outs.items()}
        kernel.visibility_device(scene, r.data_ptr(), r.shape[0], l.data_ptr(), l.shape[0], ptrs(ref), hierarchy=h)
        alone.append(ref)
    torch.cuda.synchronize()
    b = Batch(kernel)
    for scene, r, l, h, outs in jobs:
        b.add(scene, r.data_ptr(), r.shape[0], l.data_ptr(), l.shape[0], ptrs(outs), hierarchy=h)
    for submission in range(3):  # direct + capture, then graph replays
        for *_, outs in jobs:
            for v in outs.values():
                v.zero_()
        torch.cuda.synchronize()
        b.submit()
        b.wait()
        for (*_, outs), ref in zip(jobs, alone):
            same(outs, ref, KEYS + ("partial",))
    # The boulders cast shadows.
    assert (jobs[0][4]["any"] != 0).float().mean().item() > 0.01
    b.close()
    inst.close()
    flat.close()


def test_update_jobs_equal_the_plain_update_frame_after_frame(kernel, world):
    """Movers' stale cones recomputed by an update job of a batch (beside a
    full job of another scene) equal cc_visibility_update's, frame after
    frame; the batch is captured once and replayed with new stale flags."""
    import torch

    movable = np.arange(0, len(world.instances) - 1, 10, dtype=np.uint32)
    scene = kernel.scene_instanced(world.geometries, world.instances, movable)
    ico = scenes.icosphere_field(seed=5, n_spheres=12, subdivisions=3, width=80, height=45)
    other = kernel.scene(ico.meshes)
    dev = torch.device("cuda:0")
    rec = torch.from_numpy(world.receivers).to(dev)
    lig = torch.from_numpy(world.lights).to(dev)
    P, L = rec.shape[0], lig.shape[0]
    n = P * L
    plain, batched = outputs(torch, n), outputs(torch, n)
    for c in (plain, batched):
        kernel.visibility_device(scene, rec.data_ptr(), P, lig.data_ptr(), L, ptrs(c))
    orec = torch.from_numpy(ico.receivers).to(dev)
    olig = torch.from_numpy(ico.lights).to(dev)
    oref, oout = outputs(torch, orec.shape[0] * olig.shape[0]), outputs(torch, orec.shape[0] * olig.shape[0])
    kernel.visibility_device(other, orec.data_ptr(), orec.shape[0], olig.data_ptr(), olig.shape[0], ptrs(oref))
    torch.cuda.synchronize()
    stale = torch.zeros(n, dtype=torch.uint8, device=dev)
    b = Batch(kernel)
    b.add(other, orec.data_ptr(), orec.shape[0], olig.data_ptr(), olig.shape[0], ptrs(oout))
    b.add_update(scene, rec.data_ptr(), P, lig.data_ptr(), L, stale.data_ptr(), ptrs(batched))
    sizes = b.sizes()
    assert sizes["jobs"] == 2
    try:
        for frame in range(1, 4):
            boxes = scene.move(scenes.moved_placements(world, movable, frame))
            stale.zero_()
            count = kernel.stale_cones(scene, rec.data_ptr(), P, world.lights, boxes, stale.data_ptr())
            assert 0 < count < n
            solved = kernel.visibility_update(scene, rec.data_ptr(), P, lig.data_ptr(), L, stale.data_ptr(),
                                              ptrs(plain))
            assert solved == count
            oout["full"].zero_()
            torch.cuda.synchronize()
            b.submit()
            b.wait()
            same(batched, plain, KEYS)
            same(oout, oref, KEYS)
        # An update job refuses the outputs the update does not write.
        with pytest.raises(_lib.CCError):
            b.add_update(scene, rec.data_ptr(), P, lig.data_ptr(), L, stale.data_ptr(),
                         ptrs(outputs(torch, n, with_all=True)))
    finally:
        b.close()
        scene.close()
        other.close()


def test_served_requests_on_an_instanced_scene_equal_the_plain_call(kernel, world):
    inst = kernel.scene_instanced(world.geometries, world.instances)
    ico = scenes.icosphere_field(seed=8, n_spheres=6, subdivisions=3, width=64, height=36)
    flat = kernel.scene(ico.meshes)
    srv = Server(kernel, max_inflight=2, max_launch_cones=20_000)
    ids = [srv.add_scene(inst), srv.add_scene(flat)]
    reqs = []
    for k, (rec, lig) in enumerate([(world.receivers, world.lights), (ico.receivers, ico.lights[:2]),
                                    (world.receivers[1::3], world.lights[2:])]):
        rec = np.ascontiguousarray(rec)
        lig = np.ascontiguousarray(lig)
        out = {"full": np.zeros((lig.shape[0], rec.shape[0]), np.uint64),
               "any": np.zeros((lig.shape[0], rec.shape[0]), np.uint64),
               "irradiance": np.zeros((lig.shape[0], rec.shape[0]), np.float32),
               "fraction": np.zeros((lig.shape[0], rec.shape[0]), np.float32)}
        sid = ids[1] if k == 1 else ids[0]
        reqs.append((inst if k != 1 else flat, rec, lig, out, srv.submit(sid, rec, lig, out)))
    for scene, rec, lig, out, t in reqs:
        srv.wait(t)
        v = kernel.visibility(scene, rec, lig, outputs=KEYS)
        for key in KEYS:
            assert np.array_equal(out[key], getattr(v, key).reshape(lig.shape[0], rec.shape[0])), key
    srv.close()
    inst.close()
    flat.close()


def test_prefiltered_jobs_share_a_batch_with_exact_ones(kernel, world):
    """Prefiltering jobs (prefilter 4 and 8 bins; instanced with and without
    object splats, and world-space) run in the batch's second launch beside
    an exact job: each equals its prefiltered cc_visibility call alone, on the
    first submission and on graph replays."""
    import torch

    inst = kernel.scene_instanced(world.geometries, world.instances)
    ico = scenes.icosphere_field(seed=8, n_spheres=6, subdivisions=3, width=64, height=36)
    flat = kernel.scene(ico.meshes)
    specs = [(inst, world.receivers, world.lights, 8.0, True), (flat, ico.receivers, ico.lights, 0.0, True),
             (flat, ico.receivers[::3], ico.lights[:2], 4.0, True), (inst, world.receivers[::4], world.lights[1:], 8.0, False)]
    jobs = []
    for scene, rec, lig, pf, obj in specs:
        r = torch.from_numpy(np.ascontiguousarray(rec)).cuda()
        l = torch.from_numpy(np.ascontiguousarray(lig)).cuda()
        jobs.append((scene, r, l, pf, obj, outputs(torch, r.shape[0] * l.shape[0], with_all=True)))
    alone = []
    for scene, r, l, pf, obj, outs in jobs:
        ref = {k: torch.zeros_like(v) for k, v in outs.items()}
        kernel.prefilter, kernel.object_prefilter = pf, obj
        try:
            kernel.visibility_device(scene, r.data_ptr(), r.shape[0], l.data_ptr(), l.shape[0], ptrs(ref))
        finally:
            kernel.prefilter, kernel.object_prefilter = 0.0, True
        alone.append(ref)
    torch.cuda.synchronize()
    b = Batch(kernel)
    for scene, r, l, pf, obj, outs in jobs:
        kernel.object_prefilter = obj
        try:
            b.add(scene, r.data_ptr(), r.shape[0], l.data_ptr(), l.shape[0], ptrs(outs), prefilter=pf)
        finally:
            kernel.object_prefilter = True
    assert b.sizes()["jobs"] == 4
    for submission in range(3):
        for *_, outs in jobs:
            for v in outs.values():
                v.zero_()
        torch.cuda.synchronize()
        b.submit()
        b.wait()
        for (*_, outs), ref in zip(jobs, alone):
            same(outs, ref, KEYS + ("partial",))
    b.close()
    inst.close()
    flat.close()


def test_served_prefiltered_requests_equal_the_plain_call(kernel, world):
    """Prefiltering requests (cc_request.prefilter) beside exact ones, on an
    instanced and a world-space scene: each launch runs its exact jobs
    through the split path and its prefiltering jobs through the
    prefiltering kernel; every result equals the plain call's. The lighting
    cache keeps exact and prefiltered results of the same light apart."""
    inst = kernel.scene_instanced(world.geometries, world.instances)
    ico = scenes.icosphere_field(seed=8, n_spheres=6, subdivisions=3, width=64, height=36)
    flat = kernel.scene(ico.meshes)
    srv = Server(kernel, max_inflight=2, max_launch_cones=30_000)
    ids = {id(inst): srv.add_scene(inst), id(flat): srv.add_scene(flat)}
    specs = [(inst, world.receivers, world.lights, 8.0), (flat, ico.receivers, ico.lights[:2], 4.0),
             (inst, world.receivers[1::3], world.lights[2:], 0.0), (flat, ico.receivers, ico.lights[:2], 0.0)]
    reqs = []
    for scene, rec, lig, pf in specs:
        rec = np.ascontiguousarray(rec)
        lig = np.ascontiguousarray(lig)
        out = {"full": np.zeros((lig.shape[0], rec.shape[0]), np.uint64),
               "any": np.zeros((lig.shape[0], rec.shape[0]), np.uint64),
               "irradiance": np.zeros((lig.shape[0], rec.shape[0]), np.float32),
               "fraction": np.zeros((lig.shape[0], rec.shape[0]), np.float32)}
        t = srv.submit(ids[id(scene)], rec, lig, out, cache_key=5, prefilter=pf)
        reqs.append((scene, rec, lig, pf, out, t))
    for scene, rec, lig, pf, out, t in reqs:
        srv.wait(t)
        kernel.prefilter = pf
        try:
            v = kernel.visibility(scene, rec, lig, outputs=KEYS)
        finally:
            kernel.prefilter = 0.0
        for key in KEYS:
            assert np.array_equal(out[key], getattr(v, key).reshape(lig.shape[0], rec.shape[0])), (pf, key)
    with pytest.raises(_lib.CCError):
        srv.submit(ids[id(flat)], ico.receivers, ico.lights[:1], {}, hierarchy=1, prefilter=1.0)
    srv.close()
    inst.close()
    flat.close()
