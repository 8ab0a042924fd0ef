"""Error statuses of the library on a B200, each caused on the host side of
a well-formed run (nothing here faults, traps or hangs the GPU):

  * CC_ERR_TIMEOUT: a bounded wait (cc_batch_wait, cc_server_wait) that runs
    out while the work is still on the device; a later wait completes it;
  * CC_ERR_BUSY: a server whose bounded queue is full refuses a submission;
  * CC_ERR_STACK: a triangle hierarchy deeper than the walk's 64-entry stack
    is flagged (the kernel checks every push against the stack's size and
    skips the entry, so the walk stays in bounds), reported by the call and
    in the flagged cones' status words.
"""
import numpy as np
import pytest

from continuum_b200 import Batch, Server, _lib, scenes
from continuum_b200._lib import CCError

pytestmark = pytest.mark.gpu

KEYS = ("full", "any", "irradiance", "fraction")


@pytest.fixture(scope="module")
def field(kernel):
    """A mid-sized field: 640 x 360 hits, 4 lights, about 0.9 M cones (tens
    of milliseconds on the device)."""
    w = scenes.icosphere_field(seed=5, n_spheres=60, subdivisions=4, width=640, height=360)
    scene = kernel.scene(w.meshes)
    yield w, scene
    scene.close()


def test_batch_wait_times_out_then_completes(kernel, field):
    import torch

    w, scene = field
    dev = torch.device("cuda:0")
    rec = torch.from_numpy(w.receivers).to(dev)
    lig = torch.from_numpy(w.lights).to(dev)
    P, L = rec.shape[0], lig.shape[0]
    b = Batch(kernel)
    outs = []
    for _ in range(8):  # the same job eight times: several hundred milliseconds in all
        o = {k: torch.zeros(P * L, dtype=torch.int64 if k in ("full", "any") else torch.float32, device=dev)
             for k in KEYS}
        outs.append(o)
        b.add(scene, rec.data_ptr(), P, lig.data_ptr(), L, {k: v.data_ptr() for k, v in o.items()})
    b.submit(Batch.options(flags=0))
    with pytest.raises(CCError) as e:
        b.wait(timeout_ms=0)
    assert e.value.code == _lib.CC_ERR_TIMEOUT
    b.wait()
    alone = kernel.visibility(scene, w.receivers, w.lights, outputs=KEYS)
    for o in outs:
        for k in KEYS:
            got = o[k].cpu().numpy().reshape(L, P)
            want = getattr(alone, k)
            assert np.array_equal(got.view(np.uint32), np.ascontiguousarray(want).view(np.uint32)), k
    b.close()


def host_outputs(P, L):
    return {"full": np.zeros((L, P), np.uint64), "any": np.zeros((L, P), np.uint64),
            "irradiance": np.zeros((L, P), np.float32), "fraction": np.zeros((L, P), np.float32)}


def test_server_wait_times_out_then_completes(kernel, field):
    w, scene = field
    srv = Server(kernel, max_inflight=1)
    sid = srv.add_scene(scene)
    P, L = w.receivers.shape[0], w.lights.shape[0]
    outs = [host_outputs(P, L) for _ in range(4)]
    tickets = [srv.submit(sid, w.receivers, w.lights, o) for o in outs]
    with pytest.raises(CCError) as e:
        srv.wait(tickets[-1], timeout_ms=0)
    assert e.value.code == _lib.CC_ERR_TIMEOUT
    for t in tickets:  # a ticket that timed out is still known, and completes
        srv.wait(t)
    srv.close()
    alone = kernel.visibility(scene, w.receivers, w.lights, outputs=KEYS)
    for o in outs:
        for k in KEYS:
            assert np.array_equal(o[k].view(np.uint32), np.ascontiguousarray(getattr(alone, k)).view(np.uint32)), k


def test_full_server_queue_refuses_with_busy(kernel, field):
    """One launch slot and room for one queued request: of six large
    requests submitted at once, the server refuses some with CC_ERR_BUSY and
    completes every one it accepted."""
    w, scene = field
    srv = Server(kernel, max_inflight=1, max_queue=1)
    sid = srv.add_scene(scene)
    P, L = w.receivers.shape[0], w.lights.shape[0]
    accepted, refused = [], 0
    for _ in range(6):
        o = host_outputs(P, L)
        try:
            accepted.append((srv.submit(sid, w.receivers, w.lights, o), o))
        except CCError as e:
            assert e.code == _lib.CC_ERR_BUSY
            refused += 1
    assert refused >= 1 and len(accepted) >= 1
    for t, _ in accepted:
        srv.wait(t)
    st = srv.stats()
    srv.close()
    assert st["refused"] == refused and st["completed"] == len(accepted)
    alone = kernel.visibility(scene, w.receivers, w.lights, outputs=KEYS)
    for _, o in accepted:
        assert np.array_equal(o["full"], alone.full)


def deep_chain_scene(kernel, depth):
    """One mesh whose triangle hierarchy is a chain `depth` interior nodes
    deep: interior node 2j has a one-triangle leaf 2j + 1 and the next
    interior node 2j + 2 as children, every box the same large box. The walk
    pops the right (interior) child first, so its stack grows by one entry
    per level. The triangles lie far outside the cone."""
    ntris = depth + 1
    tris = np.zeros((ntris, 12), np.float32)
    for k in range(ntris):
        x = 500.0 + 2.0 * k
        tris[k, 0:3] = (x, 0.0, 0.0)
        tris[k, 4:7] = (x + 1.0, 0.0, 0.0)
        tris[k, 8:11] = (x, 1.0, 0.0)
    node = np.dtype([("lo", "<f4", 4), ("hi", "<f4", 4), ("info", "<u4", 4)])
    blas = np.zeros(2 * depth + 1, node)
    blas["lo"] = (-10.0, -10.0, -10.0, 0.0)
    blas["hi"] = (700.0, 10.0, 10.0, 0.0)
    for j in range(depth):
        blas[2 * j]["info"] = (2 * j + 1, 0, 0, 0)  # interior: children 2j + 1 and 2j + 2
        blas[2 * j + 1]["info"] = (j, 1, 0, 0)       # leaf: triangle slot j
    blas[2 * depth]["info"] = (depth, 1, 0, 0)       # the last leaf
    blas_items = np.arange(ntris, dtype=np.uint32)
    ranges = np.array([[0, ntris, 0, _lib.CC_NONE]], np.uint32)
    nodes = np.zeros(1, node)
    nodes[0]["lo"] = (-10.0, -10.0, -10.0, 0.0)
    nodes[0]["hi"] = (700.0, 10.0, 10.0, 0.0)
    nodes[0]["info"] = (0, 1, 0, 0)
    items = np.zeros(1, np.uint32)
    return kernel.scene_from_flat(tris, ranges, blas, blas_items, nodes, items)


def test_deep_hierarchy_reports_stack_overflow(kernel):
    rec = np.zeros((32, 8), np.float32)
    rec[:, 0] = np.linspace(-1.0, 1.0, 32)
    rec[:, 5] = 1.0  # on the ground, facing up
    w = scenes.box_field(grid=4)  # its light: 1 x 1 m at 4 m facing down
    shallow = deep_chain_scene(kernel, 40)
    v = kernel.visibility(shallow, rec, w.lights, outputs=KEYS + ("work",))
    assert not (v.work[..., 3] & _lib.CC_CONE_STACK).any()
    shallow.close()
    deep = deep_chain_scene(kernel, 80)
    with pytest.raises(CCError) as e:
        kernel.visibility(deep, rec, w.lights, outputs=KEYS)
    assert e.value.code == _lib.CC_ERR_STACK
    # Device pointers: the call returns at once; the flagged cones carry
    # CC_CONE_STACK in their status words.
    import torch

    dev = torch.device("cuda:0")
    n = rec.shape[0]
    work = torch.zeros(n, 4, dtype=torch.int32, device=dev)
    full = torch.zeros(n, dtype=torch.int64, device=dev)
    r = torch.from_numpy(rec).to(dev)
    l = torch.from_numpy(w.lights).to(dev)
    kernel.visibility_device(deep, r.data_ptr(), n, l.data_ptr(), 1, {"full": full.data_ptr(), "work": work.data_ptr()})
    torch.cuda.synchronize()
    status = work[:, 3].cpu().numpy().view(np.uint32)
    assert ((status & _lib.CC_CONE_STACK) != 0).all()
    deep.close()
