"""ORACLE — test infrastructure. A plain-Python restatement of the lighting
cache's page manager (crates/continuum-gpu/src/vcache.rs) for the direct
light of static lights: the checker of the library's planner (cc_planner_*,
continuum_b200/csrc/cache_plan.cpp). Used only by tests/.

Restated, citing vcache.rs:
  * PAGE / STRIDE / PAGE_TEXELS :32-35; MIN_BUDGET :52; START_BUDGET :80;
    EVICT_PER_FRAME :41, EVICT_AGE :44, EVICT_ABOVE :51, FLOOR_FRESH :55;
  * BakeModel (least squares of bake time on budget with forgetting) :1105-1160;
  * begin_frame's budget: the floor period :3005-3023, the model :3029-3048,
    the period rule :3049-3063, the frame-budget cap :3065-3079, eviction
    :3087-3092 (pages unused for EVICT_AGE frames once a quarter is resident);
  * plan :3704-3790 (requests by priority, at most `budget` of them), and
    plan_page :3928-4060 (cost = inside texels x lights; the first page always
    fits; a full pool evicts pages unused for 2 frames once a frame; jobs
    [bake-list index, texel | light << 8] light by light over the listed
    texels, inside + 1 per axis, at most 9);
  * queue_stale / evict_queued :3498-3539; free slots pop from slot 0 :1871.
Float arithmetic follows the reference's types (f32 budget and model
outputs, f64 model sums).
"""
from __future__ import annotations

import numpy as np

PAGE = 8
STRIDE = PAGE + 1
PAGE_TEXELS = STRIDE * STRIDE
EMPTY = 0xFFFFFFFF
MIN_BUDGET = np.float32(1000.0)
START_BUDGET = np.float32(8000.0)
EVICT_PER_FRAME = 2048
EVICT_AGE = 64
EVICT_ABOVE = np.float32(0.25)
FLOOR_FRESH = 120
f32 = np.float32


class BakeModel:
    def __init__(self):
        self.sums = [0.0] * 5
        self.latency = f32(1.0)
        self.cost = f32(5e-4)
        self.render = f32(0.0)

    def add(self, units, bake_ms, render_ms):
        self.render = f32(render_ms) if self.render == 0 else f32(f32(0.7) * self.render + f32(0.3) * f32(render_ms))
        if units <= 0:
            return
        u, y = float(f32(units)), float(f32(bake_ms))
        for i, x in enumerate((1.0, u, u * u, y, u * y)):
            self.sums[i] = 0.95 * self.sums[i] + x
        w, su, suu, sy, suy = self.sums
        mu, my = su / w, sy / w
        var = suu / w - mu * mu
        if w >= 4.0 and var > (0.1 * mu) * (0.1 * mu):
            self.cost = f32(min(max(f32((suy / w - mu * my) / var), f32(1e-6)), f32(1.0)))
        self.latency = f32(min(max(f32(my - float(self.cost) * mu), f32(0.0)), f32(100.0)))

    def budget(self, target):
        return f32(f32(f32(f32(target) - self.render) - self.latency) / self.cost)


class Planner:
    def __init__(self, pages, lights, bake_budget, frame_target_ms=0.0, frame_budget_ms=0.0, floor_overrun=0.25):
        self.pages, self.lights, self.bake_budget = pages, lights, bake_budget
        self.target, self.budget_ms, self.overrun = f32(frame_target_ms), f32(frame_budget_ms), f32(floor_overrun)
        self.budget = min(START_BUDGET, f32(bake_budget)) if self.target > 0 else f32(bake_budget)
        self.cap = f32(bake_budget)
        self.frame = 0
        self.periods = [f32(0)] * 3
        self.floor_period, self.floor_frame = f32(0), 0
        self.model_frame, self.latest = 0, 0
        self.model = BakeModel()
        self.map = {}
        self.slot_key = [None] * pages
        self.last_used = [0] * pages
        self.free = list(range(pages - 1, -1, -1))
        self.evict_queue = []
        self.planned, self.jobs, self.spent, self.evicted = [], [], 0, 0

    def limit(self, l):
        overrun = max(self.overrun, f32(0))
        known = self.floor_frame > 0 and self.floor_frame + FLOOR_FRESH >= self.frame
        return f32((f32(1) + overrun) * self.floor_period) if overrun > 0 and known and self.floor_period > l else l

    def begin_frame(self, period_ms=0.0, render_ms=0.0, gpu_waited=False, bake_ms=-1.0, units=0.0):
        if bake_ms >= 0 and self.frame > 0:
            self.model.add(units, bake_ms, render_ms)
            self.model_frame = self.frame - 1
            self.latest = max(self.latest, self.frame - 1)
        period = None
        if period_ms > 0:
            self.periods = [self.periods[1], self.periods[2], f32(period_ms)]
            s = sorted(self.periods)
            period = f32(period_ms) if s[0] == 0 else s[1]
        floor = min(MIN_BUDGET, f32(self.bake_budget))
        bb = f32(self.bake_budget)
        if self.target > 0 and period is not None and self.budget <= f32(1.2) * floor:
            fresh = self.floor_frame > 0 and self.floor_frame + 8 >= self.frame
            self.floor_period = f32(f32(0.8) * self.floor_period + f32(0.2) * period) if fresh else period
            self.floor_frame = self.frame
        model = self.model_frame > 0 and self.model_frame + 32 >= self.frame
        if self.target > 0 and model:
            if self.latest > 0:
                dither = f32(1.0) if self.frame % 2 == 0 else f32(0.8)
                self.budget = min(max(f32(self.model.budget(self.target) * dither), floor), bb)
        elif self.target > 0 and period is not None:
            tl = self.limit(self.target)
            if gpu_waited and period > tl:
                self.budget = f32(self.budget * f32(tl / period))
            elif period < tl:
                self.budget = f32(self.budget * f32(1.1))
            self.budget = min(max(self.budget, floor), bb)
        if self.budget_ms > 0 and self.target > 0 and period is not None:
            bm = self.limit(self.budget_ms)
            if period > bm:
                self.cap = max(f32(f32(min(self.budget, self.cap) * bm) / period), floor)
            elif period < f32(0.85) * bm:
                self.cap = min(f32(self.cap * f32(1.05)), bb)
            self.budget = min(self.budget, self.cap)
        if f32(len(self.map)) > EVICT_ABOVE * f32(self.pages):
            self.queue_stale(EVICT_AGE)
            self.evicted += self.evict_queued(EVICT_PER_FRAME, EVICT_AGE)

    def queue_stale(self, age):
        stale = [(self.last_used[s], s) for s in range(self.pages)
                 if self.slot_key[s] is not None and self.last_used[s] + age < self.frame]
        stale.sort(reverse=True)
        self.evict_queue = [s for _, s in stale]

    def evict_queued(self, count, age):
        freed = 0
        while freed < count and self.evict_queue:
            s = self.evict_queue.pop()
            if self.slot_key[s] is None or self.last_used[s] + age >= self.frame:
                continue
            del self.map[self.slot_key[s]]
            self.slot_key[s] = None
            self.free.append(s)
            freed += 1
        return freed

    def plan(self, requests):
        """requests: (key tuple, priority, (inside_x, inside_y))."""
        self.planned, self.jobs, self.spent = [], [], 0
        order = []
        for i, (key, prio, inside) in enumerate(requests):
            key = tuple(key)
            if key in self.map:
                self.last_used[self.map[key]] = self.frame
                continue
            order.append((prio, key, i))
        budget = max(int(self.budget), PAGE_TEXELS)
        order.sort()
        order = order[:budget]
        evicted_now = [False]
        for prio, key, i in order:
            if self.plan_page(key, requests[i][2], i, budget, evicted_now) == "full":
                break

    def plan_page(self, key, inside, index, budget, evicted_now):
        if key in self.map:
            return "skipped"
        inside = (min(inside[0], STRIDE), min(inside[1], STRIDE))
        if inside[0] == 0 or inside[1] == 0:
            return "skipped"
        listed = (min(inside[0] + 1, STRIDE), min(inside[1] + 1, STRIDE))
        cost = inside[0] * inside[1] * self.lights
        if self.spent + cost > budget and self.planned:
            return "full"
        if not self.free and not evicted_now[0]:
            evicted_now[0] = True
            self.queue_stale(2)
            self.evicted += self.evict_queued(EVICT_PER_FRAME, 2)
        if not self.free:
            return "full"
        slot = self.free.pop()
        self.map[key] = slot
        self.slot_key[slot] = key
        self.last_used[slot] = self.frame
        b = len(self.planned)
        self.planned.append((key, slot, index, listed))
        for l in range(self.lights):
            for y in range(listed[1]):
                for x in range(listed[0]):
                    self.jobs.append((b, (y * STRIDE + x) | (l << 8)))
        self.spent += cost
        return "planned"

    def end_frame(self):
        self.frame += 1
