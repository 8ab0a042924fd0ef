"""The served form (cc_server_*) on a B200: every request's results are the
same alone and in the mix, the lighting cache serves recoloured lights, and
admission keeps device memory under the budget."""
import numpy as np
import pytest

from continuum_b200 import Server, _lib, scenes

pytestmark = pytest.mark.gpu

KEYS = ("full", "any", "irradiance", "fraction")


def host_outputs(P, L):
    return {"full": np.zeros((L, P), np.uint64), "any": np.zeros((L, P), np.uint64),
            "irradiance": np.zeros((L, P), np.float32), "fraction": np.zeros((L, P), np.float32)}


def alone(kernel, scene, rec, lights):
    v = kernel.visibility(scene, rec, lights, outputs=KEYS)
    return {k: getattr(v, k).reshape(lights.shape[0], rec.shape[0]) for k in KEYS}


def recolour(light, rgb):
    out = light.copy()
    out[12:15] = rgb
    return out


@pytest.fixture(scope="module")
def fields(kernel):
    ws = [scenes.icosphere_field(seed=5, n_spheres=12, subdivisions=4, width=160, height=90),
          scenes.icosphere_field(seed=8, n_spheres=6, subdivisions=3, width=96, height=54),
          scenes.box_field(grid=96)]
    sc = [kernel.scene(w.meshes) for w in ws]
    yield ws, sc
    for s in sc:
        s.close()


@pytest.mark.parametrize("chunk", [None, 3000])
def test_each_request_is_the_same_alone_and_in_the_mix(kernel, fields, chunk):
    """(chunk: launches split into chunks of at most that many cones, which
    end inside requests.)"""
    ws, sc = fields
    if chunk:
        kernel.set_split_chunk(chunk)
    try:
        srv = Server(kernel, max_inflight=3, max_launch_cones=40_000)
    finally:
        kernel.set_split_chunk(1 << 25)
    ids = [srv.add_scene(s) for s in sc]
    rng = np.random.default_rng(4)
    reqs = []
    for i in range(12):
        k = i % 3
        w = ws[k]
        n = int(rng.integers(500, w.receivers.shape[0]))
        start = int(rng.integers(0, w.receivers.shape[0] - n + 1))
        rec = np.ascontiguousarray(w.receivers[start:start + n])
        pick = rng.permutation(w.lights.shape[0])[: int(rng.integers(1, w.lights.shape[0] + 1))]
        lig = np.ascontiguousarray(w.lights[pick])
        reqs.append((k, rec, lig, host_outputs(n, lig.shape[0])))
    tickets = [srv.submit(ids[k], rec, lig, out) for k, rec, lig, out in reqs]
    stats = [srv.wait(t) for t in tickets]
    s = srv.stats()
    assert s["completed"] == 12 and s["launches"] >= 2
    assert max(st["launch_requests"] for st in stats) >= 2  # requests shared launches
    for (k, rec, lig, out) in reqs:
        ref = alone(kernel, sc[k], rec, lig)
        for key in KEYS:
            assert np.array_equal(out[key], ref[key]), key
    srv.close()


def test_the_lighting_cache_serves_recoloured_lights(kernel, fields):
    ws, sc = fields
    w = ws[0]
    srv = Server(kernel)
    sid = srv.add_scene(sc[0])
    rec = w.receivers
    first = np.ascontiguousarray(w.lights[:2])
    out1 = host_outputs(rec.shape[0], 2)
    st1 = srv.wait(srv.submit(sid, rec, first, out1, cache_key=77))
    assert st1["cached_lights"] == 0
    # Light 0 recoloured (same geometry: served from the cache), light 3 new.
    second = np.ascontiguousarray(np.stack([recolour(w.lights[0], (5.0, 0.5, 0.1)), w.lights[3]]))
    out2 = host_outputs(rec.shape[0], 2)
    st2 = srv.wait(srv.submit(sid, rec, second, out2, cache_key=77))
    assert st2["cached_lights"] == 1
    ref = alone(kernel, sc[0], rec, second)
    for key in KEYS:
        assert np.array_equal(out2[key], ref[key]), key
    # Without the key nothing is served from the cache.
    out3 = host_outputs(rec.shape[0], 2)
    assert srv.wait(srv.submit(sid, rec, second, out3))["cached_lights"] == 0
    assert srv.stats()["cache_entries"] >= 3
    srv.close()


def test_admission_stays_under_the_budget(kernel, fields):
    ws, sc = fields
    w = ws[0]
    rec, lig = w.receivers, w.lights
    P, L = rec.shape[0], lig.shape[0]
    # Room for two or three requests in flight, but not for every request's
    # cached results besides: admission must evict cache entries. A launch
    # also holds 368 bytes of split-path scratch per traced cone.
    budget = P * 32 + L * 64 + L * P * (28 + 368) + P * 4 + 64 * P + (4 << 20)
    srv = Server(kernel, hbm_budget=budget, max_inflight=4)
    sid = srv.add_scene(sc[0])
    outs = [host_outputs(P, L) for _ in range(4)]
    tickets = [srv.submit(sid, rec, lig, o, cache_key=i + 1) for i, o in enumerate(outs)]
    for t in tickets:
        srv.wait(t)
    s = srv.stats()
    assert s["completed"] == 4
    assert s["peak_bytes"] <= budget
    ref = alone(kernel, sc[0], rec, lig)
    for o in outs:
        for key in KEYS:
            assert np.array_equal(o[key], ref[key]), key
    # A request larger than the whole budget is refused at submission.
    big = np.ascontiguousarray(np.concatenate([rec] * 4))
    with pytest.raises(_lib.CCError) as e:
        srv.submit(sid, big, lig, host_outputs(big.shape[0], L))
    assert e.value.code == _lib.CC_ERR_BUSY
    assert srv.stats()["refused"] == 1
    srv.close()


@pytest.mark.parametrize("ns_per_cone", [12, 0])
def test_small_requests_overtake_large_ones(kernel, fields, ns_per_cone):
    """Earliest deadline first: while one launch runs (one slot, one request
    a launch), a small request submitted just after a large one is admitted
    first, and the large one after the small one has completed; with no time
    per cone (arrival order) the small one waits for the large one. Results
    are the same either way."""
    import time

    ws, sc = fields
    w = ws[0]
    srv = Server(kernel, max_inflight=1, max_launch_cones=1, deadline_ns_per_cone=ns_per_cone)
    sid = srv.add_scene(sc[0])
    busy = np.ascontiguousarray(np.concatenate([w.receivers] * 8))
    big_rec, big_lig = w.receivers, w.lights
    small_rec, small_lig = np.ascontiguousarray(w.receivers[:500]), np.ascontiguousarray(w.lights[:1])
    outs = [host_outputs(busy.shape[0], big_lig.shape[0]), host_outputs(big_rec.shape[0], big_lig.shape[0]),
            host_outputs(500, 1)]
    t_busy = srv.submit(sid, busy, big_lig, outs[0])
    t0 = time.perf_counter()
    t_big = srv.submit(sid, big_rec, big_lig, outs[1])
    t_small = srv.submit(sid, small_rec, small_lig, outs[2])
    between_ms = 1e3 * (time.perf_counter() - t0)
    srv.wait(t_busy)
    big, small = srv.wait(t_big), srv.wait(t_small)
    if ns_per_cone:
        # The large request was admitted after the small one completed.
        assert big["queued_ms"] >= small["total_ms"]
    else:
        assert small["queued_ms"] + between_ms >= big["total_ms"]
    assert srv.stats()["launches"] == 3
    for out, rec, lig in ((outs[1], big_rec, big_lig), (outs[2], small_rec, small_lig)):
        ref = alone(kernel, sc[0], rec, lig)
        for key in KEYS:
            assert np.array_equal(out[key], ref[key]), key
    srv.close()


def test_a_slot_stays_free_of_requests_above_the_launch_limit(kernel, fields):
    """Two slots, a launch limit of 9M cones, 1 ns of deadline per cone. A
    request above the limit (a, 17.3M cones) and one within it (s, 8.6M)
    hold both slots; then a second request above the limit (b, 9.2M) and,
    12 ms later, a small one (c) queue, b with the earlier deadline. When s
    completes, c takes the slot and b keeps waiting, since a slot stays free
    of requests above the limit while a smaller one waits. (Pinned host
    buffers: a copy to pageable memory would hold the server's thread until
    the launch before it is done.)"""
    import time

    import torch

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.from_numpy(a[:0]).dtype).pin_memory()
        t.numpy()[...] = a
        return t.numpy()

    ws, sc = fields
    w = ws[0]
    lig = w.lights
    assert lig.shape[0] == 4
    srv = Server(kernel, max_inflight=2, max_launch_cones=9_000_000, deadline_ns_per_cone=1)
    sid = srv.add_scene(sc[0])
    a_rec = pinned(np.concatenate([w.receivers] * 300))   # 17.3 M cones with 4 lights
    s_rec = pinned(np.concatenate([w.receivers] * 150))   # 8.6 M cones
    b_rec = pinned(np.concatenate([w.receivers] * 160))   # 9.2 M cones
    small_rec, small_lig = pinned(w.receivers[:500]), np.ascontiguousarray(w.lights[:1])
    shapes = ((a_rec.shape[0], 4), (s_rec.shape[0], 4), (b_rec.shape[0], 4), (500, 1))
    outs = [{k: pinned(v) for k, v in host_outputs(P, L).items()} for P, L in shapes]
    # A first request, so that the server's thread is up and idle.
    srv.wait(srv.submit(sid, small_rec, small_lig, outs[3]))
    t_a = srv.submit(sid, a_rec, lig, outs[0])
    time.sleep(0.003)
    t_s = srv.submit(sid, s_rec, lig, outs[1])
    time.sleep(0.001)
    t0 = time.perf_counter()
    t_b = srv.submit(sid, b_rec, lig, outs[2])
    time.sleep(0.012)
    t_c = srv.submit(sid, small_rec, small_lig, outs[3])
    between_ms = 1e3 * (time.perf_counter() - t0)
    a, s_, b, c = (srv.wait(t) for t in (t_a, t_s, t_b, t_c))
    # c was admitted before b although b's deadline came first.
    assert c["queued_ms"] + between_ms < b["queued_ms"], (a, s_, b, c, between_ms)
    for out, r, li in ((outs[2], b_rec, lig), (outs[3], small_rec, small_lig)):
        ref = alone(kernel, sc[0], r, li)
        for key in KEYS:
            assert np.array_equal(out[key], ref[key]), key
    srv.close()


def test_the_server_trace_lists_every_launch():
    """CC_SERVER_TRACE set: the server reports its budget reservation at
    creation and one line per launch (admitted, enqueue time, retired,
    requests, cones, busy slots and the enqueue's parts) when destroyed.
    Run in a child process, where the variable is set before the server is
    made."""
    import os
    import subprocess
    import sys
    import textwrap

    code = textwrap.dedent("""
        import numpy as np
        from continuum_b200 import MaskConeKernel, Server, scenes
        w = scenes.box_field(grid=32)
        k = MaskConeKernel(0)
        sc = k.scene(w.meshes)
        srv = Server(k, hbm_budget=1 << 30, max_inflight=2)
        sid = srv.add_scene(sc)
        P, L = w.receivers.shape[0], w.lights.shape[0]
        outs = [{"full": np.zeros((L, P), np.uint64), "any": np.zeros((L, P), np.uint64),
                 "irradiance": np.zeros((L, P), np.float32), "fraction": np.zeros((L, P), np.float32)}
                for _ in range(3)]
        for t in [srv.submit(sid, w.receivers, w.lights, o) for o in outs]:
            srv.wait(t)
        launches = srv.stats()["launches"]
        srv.close()
        print("launches", launches)
    """)
    env = dict(os.environ, CC_SERVER_TRACE="1")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    launches = int(r.stdout.split("launches")[1])
    lines = [l for l in r.stderr.splitlines() if l.startswith("cc_server trace:")]
    assert any("reserved 1.00 GiB" in l for l in lines)
    rows = [l.split(":", 1)[1].split() for l in lines if "reserved" not in l and "admitted_ms" not in l]
    assert len(rows) == launches >= 1
    for row in rows:
        admitted, enqueue, retired = (float(x) for x in row[:3])
        assert len(row) == 11 and retired >= admitted and enqueue >= 0.0
    assert sum(int(row[3]) for row in rows) == 3
