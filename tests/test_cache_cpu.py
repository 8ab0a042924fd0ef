"""The lighting cache's page manager (cc_planner_*, host only) against the
oracle's restatement of vcache.rs (oracle/cache_plan.py): planning order,
budget, jobs, slots, eviction and the adaptive budget, frame by frame."""
import numpy as np
import pytest

from continuum_b200 import PageRequest, Planner
from oracle import cache_plan as ref


def run_both(frames, nlights=2, **opt):
    lib = Planner(nlights=nlights, **opt)
    orc = ref.Planner(opt.get("pages", 1 << 16), nlights, opt.get("bake_budget", 1 << 20), opt.get("frame_target_ms", 0.0),
                      opt.get("frame_budget_ms", 0.0), opt.get("floor_overrun", 0.25))
    for reqs, timing in frames:
        st = lib.frame([PageRequest(k, p, i) for k, p, i in reqs], **timing)
        units = orc.spent
        orc.begin_frame(timing.get("period_ms", 0.0), timing.get("render_ms", 0.0), timing.get("gpu_waited", False),
                        timing.get("bake_ms", -1.0), units)
        orc.plan(reqs)
        jobs, slots = lib.jobs()
        assert st["budget"] == pytest.approx(float(orc.budget), rel=0, abs=0), (st, orc.budget)
        assert st["pages_planned"] == len(orc.planned)
        assert st["spent"] == orc.spent
        assert st["resident"] == len(orc.map)
        assert st["evicted"] == orc.evicted
        assert [int(s) for s in slots] == [p[1] for p in orc.planned]
        assert jobs.shape[0] == len(orc.jobs)
        if orc.jobs:
            assert np.array_equal(jobs, np.asarray(orc.jobs, np.uint32))
        for key, slot, _, _ in orc.planned:
            assert lib.slot(key) == slot
        orc.end_frame()
        yield st, orc


def random_frames(seed, n_frames, n_keys, per_frame, timed):
    rng = np.random.default_rng(seed)
    keys = [(int(a), int(b), int(c)) for a, b, c in rng.integers(0, 50, size=(n_keys, 3))]
    for f in range(n_frames):
        pick = rng.choice(len(keys), size=per_frame, replace=True)
        reqs = [(keys[i], int(rng.integers(0, 1 << 12)), (int(rng.integers(0, 10)), int(rng.integers(0, 10))))
                for i in pick]
        timing = {}
        if timed:
            timing = {"period_ms": float(rng.uniform(6, 30)), "render_ms": float(rng.uniform(1, 6)),
                      "gpu_waited": bool(rng.integers(0, 2))}
            if f > 0 and rng.random() < 0.8:
                timing["bake_ms"] = float(rng.uniform(0.2, 12))
        yield reqs, timing


@pytest.mark.parametrize("opt", [
    dict(pages=4096, bake_budget=20000),
    dict(pages=64, bake_budget=6000),                                     # the pool fills: evictions
    dict(pages=4096, bake_budget=200000, frame_target_ms=14.0),            # the adaptive budget
    dict(pages=4096, bake_budget=200000, frame_target_ms=14.0, frame_budget_ms=11.0),
    dict(pages=256, bake_budget=50000, frame_target_ms=8.0, floor_overrun=0.0),
])
def test_planner_matches_the_restatement(opt):
    timed = opt.get("frame_target_ms", 0.0) > 0
    frames = list(random_frames(7, 60, 400, 120, timed))
    n = 0
    for _ in run_both(frames, **opt):
        n += 1
    assert n == 60


def test_model_budget_follows_the_fit():
    """Bake time = 2 ms + 1e-4 ms per cone: the model recovers latency and
    cost, and the budget becomes what fits the target after the camera passes
    (20 % less on odd frames)."""
    opt = dict(pages=1 << 14, bake_budget=1 << 22, frame_target_ms=14.0)
    rng = np.random.default_rng(3)
    keys = [(i, 0, 0) for i in range(20000)]
    frames, spent = [], 0
    lib = Planner(nlights=1, **opt)
    budgets = []
    for f in range(80):
        reqs = [PageRequest(keys[(f * 500 + i) % len(keys)], i, (8, 8)) for i in range(500)]
        bake = 2.0 + 1e-4 * spent if f > 0 else -1.0
        st = lib.frame(reqs, period_ms=16.0, render_ms=4.0, bake_ms=bake)
        spent = st["spent"]
        budgets.append((st["frame"], st["budget"]))
    # Expected: (14 - 4 - 2) / 1e-4 = 80,000 cones on even frames, 64,000 on odd.
    late = budgets[-10:]
    for frame, b in late:
        want = 80000.0 * (1.0 if frame % 2 == 0 else 0.8)
        assert b == pytest.approx(want, rel=0.02), (frame, b)


def test_first_page_always_fits_and_jobs_are_listed_light_by_light():
    lib = Planner(nlights=3, pages=16, bake_budget=100)
    st = lib.frame([PageRequest((1, 2, 3), 5, (9, 9)), PageRequest((4, 5, 6), 1, (3, 2))])
    # Priority 1 first: 3 x 2 texels x 3 lights = 18 cones; the 9 x 9 page
    # (243 cones) no longer fits the 100-cone budget.
    assert st["pages_planned"] == 1 and st["spent"] == 18
    jobs, slots = lib.jobs()
    listed = [(y * 9 + x) | (l << 8) for l in range(3) for y in range(3) for x in range(4)]
    assert jobs[:, 0].tolist() == [0] * len(listed)
    assert jobs[:, 1].tolist() == listed
    assert slots.tolist() == [0]
    # Alone, the costly page is planned all the same.
    st = lib.frame([PageRequest((1, 2, 3), 5, (9, 9))])
    assert st["pages_planned"] == 1 and st["spent"] == 243
    assert lib.slot((1, 2, 3)) == 1 and lib.slot((4, 5, 6)) == 0


def test_resident_requests_count_as_use_and_stale_pages_are_evicted():
    lib = Planner(nlights=1, pages=8, bake_budget=1 << 20)
    for i in range(8):
        lib.frame([PageRequest((i, 0, 0), 0, (8, 8))])
    # The pool is full; page 7 keeps being used, the others age.
    for _ in range(3):
        st = lib.frame([PageRequest((7, 0, 0), 0, (8, 8))])
        assert st["pages_planned"] == 0
    st = lib.frame([PageRequest((100, 0, 0), 0, (8, 8))])
    # A full pool evicts pages unused for 2 frames (all but page 7), slot 0 first in line.
    assert st["pages_planned"] == 1 and st["evicted"] == 7
    assert lib.slot((7, 0, 0)) == 7 and lib.slot((100, 0, 0)) >= 0
    assert lib.slot((0, 0, 0)) == -1


def test_invalid_options_are_rejected():
    from continuum_b200._lib import CCError
    with pytest.raises(CCError):
        Planner(nlights=0)
    with pytest.raises(CCError):
        Planner(nlights=1, pages=0)
    with pytest.raises(CCError):
        Planner(nlights=1, bake_budget=0)
