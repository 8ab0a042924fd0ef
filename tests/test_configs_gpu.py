"""Every workload at its real size on a B200, against the oracle.

The small plain workload (65,536 cones) and the plain workload at scale
(3,686,400 cones over 3.07 M triangles) are checked cone for cone; the
batched workload (64 jobs, 98.9 M cones), the served workload (8 resident
scenes) and the instanced world (1 M instances, before and after moving
frames) on evenly strided samples of every checked job, request or frame.
Each is held to the parity bar (oracle/parity.py) against the FP32 oracle,
and its error against the FP64 oracle is printed beside it (`pytest -s`).
These follow the reference's own full-size checks, in which every receiver
of the run is compared (crates/continuum-gltf/tests/gpu.rs:294-337,
experiments/room3d/src/bin/m2_gate1.rs)."""
import json

import numpy as np
import pytest

from continuum_b200 import Batch, Server, _lib, scenes
from oracle.oracle import OracleScene
from oracle.parity import check_against

pytestmark = pytest.mark.gpu

KEYS = ("full", "any", "irradiance", "fraction")


def device_solve(kernel, scene, rec, lights, torch, dev, work=False):
    P, L = rec.shape[0], lights.shape[0]
    C = P * L
    outs = {"full": torch.empty(C, dtype=torch.int64, device=dev), "any": torch.empty(C, dtype=torch.int64, device=dev),
            "irradiance": torch.empty(C, device=dev), "fraction": torch.empty(C, device=dev),
            "partial": torch.empty(C, 64, device=dev)}
    if work:
        outs["work"] = torch.empty(C, 4, dtype=torch.int32, device=dev)
    r = torch.from_numpy(np.ascontiguousarray(rec)).to(dev)
    l = torch.from_numpy(np.ascontiguousarray(lights)).to(dev)
    kernel.visibility_device(scene, r.data_ptr(), P, l.data_ptr(), L, {k: v.data_ptr() for k, v in outs.items()})
    torch.cuda.synchronize(dev)
    return outs


def to_host(outs, ids=None):
    res = {}
    for k in KEYS:
        a = outs[k].reshape(-1).cpu().numpy()
        if ids is not None:
            a = a[np.asarray(ids, np.int64)]
        res[k] = a.view(np.uint64) if k in ("full", "any") else a
    return res


def rows(partial, ids=None):
    import torch

    def get(pos):
        cones = np.asarray(pos, np.int64) if ids is None else np.asarray(ids, np.int64)[np.asarray(pos, np.int64)]
        return partial[torch.from_numpy(cones).to(partial.device)].cpu().numpy()
    return get


def strided(total, n):
    if n >= total:
        return np.arange(total, dtype=np.uint64)
    return np.arange(0, total, total // n, dtype=np.uint64)[:n]


def bitwise(a, b):
    """Per element: the same bits (mask words as integers, floats as bits)."""
    a, b = np.asarray(a), np.asarray(b)
    if a.dtype == np.float32:
        return a.view(np.uint32) == b.view(np.uint32)
    return a == b


def report(name, rep):
    """The bar against the oracle with the library's summation (every
    disagreeing bit traced), and against the reference's own summation every
    disagreeing bit traced to coverage within rounding of a threshold."""
    print(f"\n{name}: {json.dumps(rep)}")
    assert rep["untraced_bits"] == 0, rep
    assert rep["meets_bar"], rep
    assert rep["reference_summation"]["untraced_bits"] == 0, rep


@pytest.fixture(scope="module")
def torch_dev():
    import torch

    return torch, torch.device("cuda", 0)


def test_small_plain_every_cone(kernel, torch_dev):
    torch, dev = torch_dev
    w = scenes.box_field(seed=1, grid=256)
    scene = kernel.scene(w.meshes)
    outs = device_solve(kernel, scene, w.receivers, w.lights, torch, dev)
    scene.close()
    osc = OracleScene(w.meshes)
    rep = check_against(osc, w.receivers, w.lights, to_host(outs), rows(outs["partial"]))
    osc.close()
    assert rep["cones"] == 65536
    report("small plain", rep)


def test_plain_at_scale_every_cone(kernel, torch_dev):
    torch, dev = torch_dev
    w = scenes.icosphere_field(seed=2)
    scene = kernel.scene(w.meshes)
    outs = device_solve(kernel, scene, w.receivers, w.lights, torch, dev)
    scene.close()
    osc = OracleScene(w.meshes)
    rep = check_against(osc, w.receivers, w.lights, to_host(outs), rows(outs["partial"]))
    osc.close()
    assert rep["cones"] == 3_686_400
    report("plain at scale", rep)


def test_batched_jobs_sampled(kernel, torch_dev):
    """Every 8th job of the 64-job batch, 8,192 strided cones each: the
    batched results equal the job solved alone, and meet the bar."""
    torch, dev = torch_dev
    jobs = scenes.batch_jobs(seed=3, njobs=64)
    sc = [kernel.scene(w.meshes) for w in jobs]
    rec = [torch.from_numpy(w.receivers).to(dev) for w in jobs]
    lig = [torch.from_numpy(w.lights).to(dev) for w in jobs]
    outs = []
    b = Batch(kernel)
    for s_, r, l in zip(sc, rec, lig):
        C = r.shape[0] * l.shape[0]
        o = {"full": torch.empty(C, dtype=torch.int64, device=dev), "any": torch.empty(C, dtype=torch.int64, device=dev),
             "irradiance": torch.empty(C, device=dev), "fraction": torch.empty(C, device=dev)}
        outs.append(o)
        b.add(s_, r.data_ptr(), r.shape[0], l.data_ptr(), l.shape[0], {k: v.data_ptr() for k, v in o.items()})
    b.submit()
    b.wait()
    b.close()
    reps = []
    for j in range(0, len(jobs), 8):
        C = rec[j].shape[0] * lig[j].shape[0]
        ids = strided(C, 8192)
        gpu = to_host(outs[j], ids)
        alone = device_solve(kernel, sc[j], jobs[j].receivers, jobs[j].lights, torch, dev)
        solo = to_host(alone, ids)
        for k in KEYS:
            assert bitwise(gpu[k], solo[k]).all(), (j, k)
        osc = OracleScene(jobs[j].meshes)
        reps.append(check_against(osc, jobs[j].receivers, jobs[j].lights, gpu, rows(alone["partial"], ids),
                                  cone_ids=ids))
        osc.close()
    for s_ in sc:
        s_.close()
    for j, rep in zip(range(0, len(jobs), 8), reps):
        report(f"batched job {j}", rep)


def test_served_requests_sampled(kernel, torch_dev):
    """Twelve requests of the serving workload through the request loop
    together; every 3rd request's results, 8,192 strided cones each, equal
    the request solved alone and meet the bar."""
    torch, dev = torch_dev
    pool = scenes.served_scenes(seed=4)
    sc = [kernel.scene(p.meshes) for p in pool]
    reqs = scenes.served_requests(pool, 12, seed=5)
    srv = Server(kernel, hbm_budget=16 << 30, max_inflight=4)
    ids_ = [srv.add_scene(s_) for s_ in sc]
    outs, tickets = [], []
    for si, pi, l in reqs:
        P, L = pool[si].poses[pi].shape[0], l.shape[0]
        o = {"full": np.zeros((L, P), np.uint64), "any": np.zeros((L, P), np.uint64),
             "irradiance": np.zeros((L, P), np.float32), "fraction": np.zeros((L, P), np.float32)}
        outs.append(o)
        tickets.append(srv.submit(ids_[si], pool[si].poses[pi], l, o, cache_key=1 + si * 16 + pi))
    for t in tickets:
        srv.wait(t)
    srv.close()
    oscenes = {}
    for i in range(0, len(reqs), 3):
        si, pi, l = reqs[i]
        recv = pool[si].poses[pi]
        C = recv.shape[0] * l.shape[0]
        ids = strided(C, 8192)
        gpu = {k: outs[i][k].reshape(-1)[ids.astype(np.int64)] for k in KEYS}
        alone = device_solve(kernel, sc[si], recv, l, torch, dev)
        solo = to_host(alone, ids)
        for k in KEYS:
            assert bitwise(gpu[k], solo[k]).all(), (i, k)
        if si not in oscenes:
            oscenes[si] = OracleScene(pool[si].meshes)
        report(f"served request {i}", check_against(oscenes[si], recv, l, gpu, rows(alone["partial"], ids),
                                                     cone_ids=ids))
    for o in oscenes.values():
        o.close()
    for s_ in sc:
        s_.close()


def test_instanced_world_sampled(kernel, torch_dev):
    """The 1 M-instance world: a full solve, then two frames in which 1% of
    the instances move and only the stale cones are recomputed; 65,536
    strided cones of the cached results meet the bar against the oracle's
    world before and after the moves."""
    torch, dev = torch_dev
    w = scenes.instanced_world(seed=5)
    movable = np.arange(0, len(w.instances) - 1, 100, dtype=np.uint32)
    scene = kernel.scene_instanced(w.geometries, w.instances, movable)
    P, L = w.receivers.shape[0], w.lights.shape[0]
    C = P * L
    cache = device_solve(kernel, scene, w.receivers, w.lights, torch, dev)
    osc = OracleScene.instanced(w.geometries, w.instances, movable)
    ids = strided(C, 65536)
    report("instanced full solve", check_against(osc, w.receivers, w.lights, to_host(cache, ids),
                                                 rows(cache["partial"], ids), cone_ids=ids))
    rec = torch.from_numpy(w.receivers).to(dev)
    lig = torch.from_numpy(w.lights).to(dev)
    stale = torch.empty(C, dtype=torch.uint8, device=dev)
    ptrs = {k: cache[k].data_ptr() for k in KEYS}
    for f in range(2):
        pl = scenes.moved_placements(w, movable, f)
        boxes = scene.move(pl)
        kernel.stale_cones(scene, rec.data_ptr(), P, w.lights, boxes, stale.data_ptr())
        kernel.visibility_update(scene, rec.data_ptr(), P, lig.data_ptr(), L, stale.data_ptr(), ptrs)
    osc.move(pl)
    # The cache equals a full solve of the moved world wherever the walk cap
    # did not stop the cone (a capped cone's result depends on its walk, which
    # a move elsewhere may change without making the cone stale).
    fresh = device_solve(kernel, scene, w.receivers, w.lights, torch, dev, work=True)
    gpu = to_host(cache, ids)
    solo = to_host(fresh, ids)
    capped = (fresh["work"][:, 3].cpu().numpy()[ids.astype(np.int64)] & _lib.CC_CONE_CAPPED) != 0
    for k in KEYS:
        assert bitwise(gpu[k], solo[k])[~capped].all(), k
    report("instanced after two moving frames", check_against(osc, w.receivers, w.lights, solo,
                                                               rows(fresh["partial"], ids), cone_ids=ids))
    osc.close()
    scene.close()
