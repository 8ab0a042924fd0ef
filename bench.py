"""Benchmark: cone-visibility queries per second on the plain-at-scale workload.

One step = one visibility solve of every (shading point, light) cone of the
plain-at-scale workload: 150 displaced icospheres (subdivision 5, 3,072,002
triangles with the ground quad), four lights (2 x 1 and 4 x 4 m rects, disks
of radius 0.5 and 1.5 m as one-sided sphere lights), and the 921,600 primary
hits of a 1280 x 720 camera: 3,686,400 cones. Synthetic, seeded data.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

The CUDA arm prints one JSON line with the device-resident throughput
(`value`), the end-to-end throughput through the C ABI with host buffers
(`e2e`), the dominant kernel's roofline, timed CPU baselines (the oracle's
FP32 restatement of the reference's GPU path on every host core, and its
restatement of the reference's CPU path on one and on every core), the SM
clocks seen during the timed region and the kernel launch count. Beside it:
the small plain workload's line (65,536 cones), the batched, served,
instanced, lighting-cache and sky forms, and an untimed accuracy report of
every workload against the oracle (FP32 for the parity bar, FP64 for the
error). The reference arm times the reference's algorithm on the host cores
(the reference is Rust + WGSL and cannot be built or run here; its FP32
restatement in oracle/ stands in for it) and loads nothing of this library:
its inputs come from the oracle's own camera pass.
Under torchrun each rank solves its own copy of the workload on its own GPU
(weak scaling); `value` is the whole job's cones per second over the slowest
rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cone visibility queries/s (plain vs batched/served), p50/p99 latency, 1 B200"
UNIT = "cones/s"
WORKLOAD = "plain at scale: 150 displaced icospheres (3,072,002 tris), 4 lights, 1280x720 primary hits"
NODE_BYTES = 48  # reference NodeGpu (hierarchy.rs:68-76)
TRI_BYTES = 48   # three vec4 vertices (hierarchy.rs:12-13)


# The full plain workload's cones per step, and the DRAM bytes of one
# packet-pass launch over them as ncu measured them (1.475 GB read + 1.453 GB
# written, 39.19 ms).
FULL_CONES = 3_686_400
PACKET_PASS_DRAM_BYTES = 1_474_594_048 + 1_453_315_584


def workload(points: int = 0, caster: str = "library"):
    """The plain-at-scale workload. caster "oracle": the receivers come from
    the oracle's camera pass (the same receivers, bit for bit), so that the
    reference arm never loads this library."""
    from continuum_b200 import scenes

    if caster == "oracle":
        from oracle.oracle import OracleScene

        w = scenes.icosphere_field(seed=2, with_receivers=False)
        osc = OracleScene(w.meshes)
        rec, hit = osc.primary_hits(w.camera, *w.size)
        osc.close()
        w.receivers = np.ascontiguousarray(rec[hit.astype(bool)])
    else:
        w = scenes.icosphere_field(seed=2)
    if points and points < w.receivers.shape[0]:
        width, height = w.size
        if w.receivers.shape[0] == width * height:
            # Whole image rows, evenly spaced: neighbours stay neighbours.
            rows = max(1, points // width)
            img = w.receivers.reshape(height, width, 8)
            w.receivers = np.ascontiguousarray(img[:: max(1, height // rows)][:rows].reshape(-1, 8))
        else:
            stride = w.receivers.shape[0] // points
            w.receivers = np.ascontiguousarray(w.receivers[::stride][:points])
    return w


def config(n_gpus: int, w) -> dict:
    return {"workload": WORKLOAD, "form": "plain", "points": int(w.receivers.shape[0]),
            "lights": int(w.lights.shape[0]), "cones_per_step": int(w.receivers.shape[0] * w.lights.shape[0]),
            "triangles": int(w.ntris), "hierarchy": "triangles", "exact": True,
            "l2": "flushed between timed steps (256 MB write); scene 200 MB > 126 MB L2",
            "parallelism": f"replica x{n_gpus}" if n_gpus > 1 else "single GPU"}


def cpu_threads() -> int:
    return max(1, len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1))


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_path_baseline(w, oscene, light_ids, max_points: int = 0, repeats: int = 5) -> dict:
    """The reference's CPU path (cone3 + coverage + the leaf-4 BVH of bvh.rs,
    Receiver::masked; oracle/ restates it) timed on the host cores as the
    reference times it: one thread, and every thread taking rows in chunks of
    64 (par_map), best of `repeats` after one warm run, the BVH's build timed
    apart. Rect lights only (the reference's CPU path has no sphere lights);
    `max_points` > 0 takes an evenly strided sample of the receivers."""
    rec = w.receivers
    if max_points and rec.shape[0] > max_points:
        rec = np.ascontiguousarray(rec[:: rec.shape[0] // max_points][:max_points])
    t0 = time.perf_counter()
    bvh = oscene.cpu_bvh()
    build_ms = (time.perf_counter() - t0) * 1e3
    lights9 = [np.concatenate([w.lights[l][0:3], w.lights[l][4:7], w.lights[l][8:11]]) for l in light_ids]
    out = {"kind": "port", "code": "restatement of the reference's CPU path (cone3.rs, coverage.rs, bvh.rs; "
                                   "Receiver::masked), not the reference binary",
           "lights": [int(l) for l in light_ids], "points": int(rec.shape[0]),
           "cones": int(rec.shape[0] * len(light_ids)), "bvh_build_ms": build_ms, "cpu_model": cpu_model()}
    for key, threads in (("threads_1", 1), ("threads_all", cpu_threads())):
        best = None
        for rep in range(repeats + 1):
            t0 = time.perf_counter()
            for l9 in lights9:
                oscene.cpu_masked_with(bvh, rec, l9, threads=threads)
            dt = time.perf_counter() - t0
            if rep and (best is None or dt < best):
                best = dt
        out[key] = {"value": out["cones"] / best, "unit": UNIT, "threads": threads, "seconds": best}
    out["cores"] = cpu_threads()
    bvh.close()
    return out


def cpu_sample(w, target_seconds: float, offset: int = 0, oscene=None):
    """Times the oracle (FP32, all host threads) on a strided sample of cones
    sized for about `target_seconds` of wall time. Returns (cones/s, cones, threads)."""
    from oracle.oracle import OracleScene

    threads = cpu_threads()
    scene = oscene if oscene is not None else OracleScene(w.meshes)
    total = w.receivers.shape[0] * w.lights.shape[0]
    probe = np.arange(offset % 97, total, max(1, total // 16384), dtype=np.uint64)[:16384]
    t0 = time.perf_counter()
    scene.visibility(w.receivers, w.lights, cone_ids=probe, threads=threads, partial=False)
    rate = len(probe) / max(time.perf_counter() - t0, 1e-6)
    n = int(min(total, max(4096, rate * target_seconds)))
    stride = max(1, total // n)
    ids = np.arange(offset % stride, total, stride, dtype=np.uint64)[:n]
    t0 = time.perf_counter()
    scene.visibility(w.receivers, w.lights, cone_ids=ids, threads=threads, partial=False)
    dt = time.perf_counter() - t0
    if oscene is None:
        scene.close()
    return len(ids) / dt, len(ids), threads, dt


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in getattr(self, "lines", []):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, val in zip(names, parts[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(x: float, world: int, device) -> float:
    """The largest of every rank's `x` (all ranks call it, in the same order);
    x itself with one rank. Each rank of a multi-GPU run solves its own replica
    of the workload, so the job's time is its slowest rank's."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(cones_per_rank: int, steps: int, world: int, slowest_seconds: float) -> float:
    """Whole-job cones/s: every rank's cones over the slowest rank's time."""
    return world * cones_per_rank * steps / slowest_seconds


def timed_steps(torch, dev, stream, flush, fn, warmup, steps):
    """Device milliseconds of `steps` calls of fn on `stream` (CUDA events,
    L2 flushed before each), after `warmup` untimed calls."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for e0, e1 in ev:
        flush.zero_()
        e0.record(stream)
        fn()
        e1.record(stream)
    torch.cuda.synchronize(dev)
    return [e0.elapsed_time(e1) for e0, e1 in ev]


def solve_on_device(kernel, scene, rec, lig, dev, stream, partial: bool = True, work: bool = False) -> dict:
    """One untimed plain solve with every output on the device (for checks)."""
    import torch

    P, L = rec.shape[0], lig.shape[0]
    C = P * L
    outs = {"full": torch.empty(C, dtype=torch.int64, device=dev), "any": torch.empty(C, dtype=torch.int64, device=dev),
            "irradiance": torch.empty(C, device=dev), "fraction": torch.empty(C, device=dev)}
    if partial:
        outs["partial"] = torch.empty(C, 64, device=dev)
    if work:
        outs["work"] = torch.empty(C, 4, dtype=torch.int32, device=dev)
    kernel.visibility_device(scene, rec.data_ptr(), P, lig.data_ptr(), L, {k: v.data_ptr() for k, v in outs.items()},
                             stream=stream.cuda_stream)
    torch.cuda.synchronize(dev)
    return outs


def host_results(outs: dict, ids=None) -> dict:
    """Device results (full, any, irradiance, fraction) as host arrays, for
    every cone or the `ids` subset."""
    import torch

    sel = None if ids is None else torch.from_numpy(np.asarray(ids, np.int64)).to(outs["full"].device)
    res = {}
    for k in ("full", "any", "irradiance", "fraction"):
        v = outs[k].reshape(-1)
        v = v if sel is None else v[sel]
        a = v.cpu().numpy()
        res[k] = a.view(np.uint64) if k in ("full", "any") else a
    return res


def partial_rows(partial, ids=None):
    """A function giving the device coverages (C, 64) of positions into `ids`
    (or of cones), as the oracle's trace asks for them."""
    import torch

    def rows(pos):
        cones = np.asarray(pos, np.int64) if ids is None else np.asarray(ids, np.int64)[np.asarray(pos, np.int64)]
        return partial[torch.from_numpy(cones).to(partial.device)].cpu().numpy()
    return rows


def same_bits(a, b) -> np.ndarray:
    """Per element: the same bits (mask words as integers, floats as bits)."""
    a, b = np.asarray(a), np.asarray(b)
    if a.dtype == np.float32:
        return a.view(np.uint32) == b.view(np.uint32)
    return a == b


def strided_ids(total: int, n: int, offset: int = 0) -> np.ndarray:
    """At most n cone numbers evenly strided over [0, total)."""
    if n <= 0 or n >= total:
        return np.arange(total, dtype=np.uint64)
    stride = total // n
    return np.arange(offset % stride, total, stride, dtype=np.uint64)[:n]


def plain_accuracy(kernel, scene, oscene, receivers, lights, dev, stream, max_cones: int = 0,
                   label: str = "every cone") -> dict:
    """The accuracy report of one plain solve (untimed) against the oracle:
    every cone, or an evenly strided sample of `max_cones`."""
    import torch

    from oracle.parity import check_against

    rec = torch.from_numpy(np.ascontiguousarray(receivers)).to(dev)
    lig = torch.from_numpy(np.ascontiguousarray(lights)).to(dev)
    C = rec.shape[0] * lig.shape[0]
    outs = solve_on_device(kernel, scene, rec, lig, dev, stream)
    ids = None if not max_cones or max_cones >= C else strided_ids(C, max_cones)
    gpu = host_results(outs, ids)
    t0 = time.perf_counter()
    rep = check_against(oscene, receivers, lights, gpu, partial_rows(outs["partial"], ids), cone_ids=ids,
                        threads=cpu_threads(), sample=label if ids is None else f"{len(ids)} strided cones of {C}")
    rep["oracle_seconds"] = time.perf_counter() - t0
    del outs
    return rep


def merge_reports(reports: list, sample: str) -> dict:
    """One accuracy report over several checked parts (jobs, requests)."""
    n = sum(r["cones"] for r in reports)
    out = {"cones": n, "sample": sample, "parts": len(reports),
           "word_agreement": sum(r["word_agreement"] * r["cones"] for r in reports) / max(n, 1),
           "max_dfraction": max((r["max_dfraction"] or 0.0) for r in reports) if reports else None,
           "max_dirradiance_rel": max((r["max_dirradiance_rel"] or 0.0) for r in reports) if reports else None,
           "mismatched_cones": sum(r["mismatched_cones"] for r in reports),
           "untraced_bits": sum(max(r["untraced_bits"], 0) for r in reports)
           if all(r["untraced_bits"] >= 0 for r in reports) else -1,
           "meets_bar": all(r["meets_bar"] for r in reports)}
    refs = [r["reference_summation"] for r in reports if "reference_summation" in r]
    if refs:
        m = sum(r["cones"] for r in reports if "reference_summation" in r)
        out["reference_summation"] = {
            "word_agreement": sum(x["word_agreement"] * r["cones"] for x, r in zip(refs, reports)) / max(m, 1),
            "mismatched_cones": sum(x["mismatched_cones"] for x in refs),
            "untraced_bits": sum(max(x["untraced_bits"], 0) for x in refs)
            if all(x["untraced_bits"] >= 0 for x in refs) else -1,
            "max_dfraction": max(x["max_dfraction"] for x in refs),
            "cones_dfraction_over_1e-3": sum(x["cones_dfraction_over_1e-3"] for x in refs),
            "exact_sums_word_agreement": {
                k: sum(x["exact_sums_word_agreement"][k] * r["cones"] for x, r in zip(refs, reports)) / max(m, 1)
                for k in ("reference_summation", "library")}}
    errs = [r["fp64_max_abs_err"] for r in reports if "fp64_max_abs_err" in r]
    if errs:
        out["fp64_max_abs_err"] = {k: max(e.get(k, 0.0) for e in errs) for k in errs[0]
                                   if k not in ("word_agreement", "cones_dfraction_over_1e-3")}
        out["fp64_max_abs_err"]["cones_dfraction_over_1e-3"] = sum(e.get("cones_dfraction_over_1e-3", 0) for e in errs)
        out["fp64_max_abs_err"]["word_agreement"] = min(e["word_agreement"] for e in errs)
    return out


def small_leg(args, kernel, dev, stream, flush) -> dict:
    """The small plain workload (the ground and 64 boxes, 770 triangles; one
    1 x 1 m rect light at 4 m; 256 x 256 receivers on the ground): 65,536
    cones per step, device-timed (CUDA events, L2 flushed) and end to end
    through cc_visibility with pinned host buffers; beside it the reference's
    CPU path and the restatement of its GPU path on the host cores, and the
    accuracy of every cone against the oracle (FP32 and FP64)."""
    import ctypes as Cc

    import torch

    from continuum_b200 import _lib, scenes
    from oracle.oracle import OracleScene

    w = scenes.box_field(seed=1, grid=256)
    scene = kernel.scene(w.meshes)
    P, L = w.receivers.shape[0], w.lights.shape[0]
    C = P * L
    rec = torch.from_numpy(w.receivers).to(dev)
    lig = torch.from_numpy(w.lights).to(dev)
    outs = {"full": torch.empty(C, dtype=torch.int64, device=dev), "any": torch.empty(C, dtype=torch.int64, device=dev),
            "irradiance": torch.empty(C, device=dev), "fraction": torch.empty(C, device=dev)}
    ptrs = {k: v.data_ptr() for k, v in outs.items()}

    def step():
        kernel.visibility_device(scene, rec.data_ptr(), P, lig.data_ptr(), L, ptrs, stream=stream.cuda_stream)

    steps = max(3, args.steps)
    ms = float(np.mean(timed_steps(torch, dev, stream, flush, step, max(3, args.warmup), steps)))
    rec_h = torch.from_numpy(w.receivers).pin_memory().numpy()
    lig_h = np.ascontiguousarray(w.lights)
    host_out = {k: torch.empty(C, dtype=dt).pin_memory().numpy() for k, dt in
                (("full", torch.int64), ("any", torch.int64), ("irradiance", torch.float32), ("fraction", torch.float32))}
    opt = kernel.options()
    o = _lib.Outputs(host_out["full"].ctypes.data, host_out["any"].ctypes.data, None,
                     host_out["irradiance"].ctypes.data, host_out["fraction"].ctypes.data, None)

    def e2e_step():
        _lib.check(_lib.load().cc_visibility(kernel.handle, scene.handle, rec_h.ctypes.data, P, lig_h.ctypes.data, L,
                                             Cc.byref(opt), Cc.byref(o), None))

    for _ in range(3):
        e2e_step()
    t0 = time.perf_counter()
    for _ in range(steps):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / steps
    out = {"workload": "small plain: a 40 x 40 m ground quad and 64 boxes (770 triangles), one 1 x 1 m one-sided rect "
                       "light at 4 m facing down, 256 x 256 receivers on the ground over [-10, 10]^2",
           "cones_per_step": C, "triangles": int(w.ntris), "steps": steps,
           "value": C / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
           "timing": "CUDA events; L2 flushed between steps (the scene is 60 KB: cache-resident)",
           "e2e": {"value": C / e2e_s, "unit": UNIT, "ms_per_step": e2e_s * 1e3,
                   "h2d_bytes_per_step": int(rec_h.nbytes + lig_h.nbytes),
                   "d2h_bytes_per_step": int(sum(v.nbytes for v in host_out.values()) + 8),
                   "path": "cc_visibility with host buffers (pinned), scene resident, wall clock"}}
    oscene = OracleScene(w.meshes)
    if not args.no_cpu_baseline:
        rate, n, threads, dt = cpu_sample(w, target_seconds=args.cpu_seconds, oscene=oscene)
        out["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"{n} strided cones of {C} ({dt:.2f} s wall); FP32 restatement of the "
                                         "reference's GPU path (oracle/)"}
    if not args.no_cpu_path:
        out["cpu_path"] = cpu_path_baseline(w, oscene, [0])
    if not args.no_accuracy:
        out["accuracy"] = plain_accuracy(kernel, scene, oscene, w.receivers, w.lights, dev, stream)
    oscene.close()
    scene.close()
    return out


def batched_leg(args, kernel, dev, stream, flush) -> dict:
    """The batching workload (64 jobs of uneven scene, light and point counts):
    cones/s of one batched submission (autotuned, replayed from a CUDA graph)
    beside the plain path called once per job, both device-timed with CUDA
    events and the L2 flushed between steps."""
    import torch

    from continuum_b200 import Batch, _lib, scenes
    from continuum_b200.kernel import kernel_times

    jobs = scenes.batch_jobs(seed=3, njobs=args.batch_jobs)
    sc = [kernel.scene(w.meshes) for w in jobs]
    rec = [torch.from_numpy(w.receivers).to(dev) for w in jobs]
    lig = [torch.from_numpy(w.lights).to(dev) for w in jobs]
    cones = [r.shape[0] * l.shape[0] for r, l in zip(rec, lig)]
    outs = [{"full": torch.empty(n, dtype=torch.int64, device=dev), "any": torch.empty(n, dtype=torch.int64, device=dev),
             "irradiance": torch.empty(n, device=dev), "fraction": torch.empty(n, device=dev)} for n in cones]
    ptrs = [{k: v.data_ptr() for k, v in o.items()} for o in outs]
    total = int(sum(cones))

    # The autotuner runs on a sample of the same jobs (every 16th point).
    sample_rec = [r[::16].contiguous() for r in rec]
    sample_out = [{k: torch.empty(max(1, sr.shape[0] * l.shape[0]), dtype=v.dtype, device=dev) for k, v in o.items()}
                  for sr, l, o in zip(sample_rec, lig, outs)]
    tb = Batch(kernel)
    for s_, sr, l, so in zip(sc, sample_rec, lig, sample_out):
        tb.add(s_, sr.data_ptr(), sr.shape[0], l.data_ptr(), l.shape[0], {k: v.data_ptr() for k, v in so.items()})
    best, tune_ms = tb.tune(reps=2)
    tb.close()
    del sample_rec, sample_out

    b = Batch(kernel)
    for s_, r, l, p in zip(sc, rec, lig, ptrs):
        b.add(s_, r.data_ptr(), r.shape[0], l.data_ptr(), l.shape[0], p)

    def batched():
        b.submit(best, stream=stream.cuda_stream)

    def plain():
        for s_, r, l, p in zip(sc, rec, lig, ptrs):
            kernel.visibility_device(s_, r.data_ptr(), r.shape[0], l.data_ptr(), l.shape[0], p,
                                     stream=stream.cuda_stream)

    steps = max(1, min(args.steps, args.batch_steps))
    # The first submission runs directly and captures the graph; later ones replay it.
    batched_ms = timed_steps(torch, dev, stream, flush, batched, 2, steps)
    b.wait()
    acc = None
    if not args.no_accuracy:
        # Untimed: every 8th job's batched results (a strided sample of its
        # cones) against the oracle, and against the plain path's.
        from oracle.oracle import OracleScene
        from oracle.parity import check_against

        reports, same = [], True
        for j in range(0, len(jobs), 8):
            ids = strided_ids(cones[j], args.accuracy_cones // 8)
            gpu = host_results(outs[j], ids)
            alone = solve_on_device(kernel, sc[j], rec[j], lig[j], dev, stream)
            solo = host_results(alone, ids)
            same = same and all(same_bits(gpu[k], solo[k]).all() for k in gpu)
            osc = OracleScene(jobs[j].meshes)
            reports.append(check_against(osc, jobs[j].receivers, jobs[j].lights, gpu,
                                         partial_rows(alone["partial"], ids), cone_ids=ids, threads=cpu_threads()))
            osc.close()
            del alone
        acc = merge_reports(reports, f"every 8th job ({len(reports)} jobs), at most "
                                     f"{args.accuracy_cones // 8} strided cones each")
        acc["batched_equals_plain"] = bool(same)
    plain_ms = timed_steps(torch, dev, stream, flush, plain, 1, steps)
    kernel_times(kernel)
    b.close()
    # The gain by job size: each class's jobs batched alone against the same
    # jobs through the plain path one at a time (same options, same timing).
    classes = []
    bounds = [(0, 100_000, "under 100k cones"), (100_000, 1_000_000, "100k-1M cones"),
              (1_000_000, 1 << 62, "1M cones or more")]
    for lo, hi, name in bounds:
        members = [j for j, c in enumerate(cones) if lo <= c < hi]
        if not members:
            continue
        cb = Batch(kernel)
        for j in members:
            cb.add(sc[j], rec[j].data_ptr(), rec[j].shape[0], lig[j].data_ptr(), lig[j].shape[0], ptrs[j])

        def class_batched():
            cb.submit(best, stream=stream.cuda_stream)

        def class_plain():
            for j in members:
                kernel.visibility_device(sc[j], rec[j].data_ptr(), rec[j].shape[0], lig[j].data_ptr(),
                                         lig[j].shape[0], ptrs[j], stream=stream.cuda_stream)

        cbt = float(np.mean(timed_steps(torch, dev, stream, flush, class_batched, 2, steps)))
        cb.wait()
        cpt = float(np.mean(timed_steps(torch, dev, stream, flush, class_plain, 1, steps)))
        kernel_times(kernel)
        cb.close()
        n = int(sum(cones[j] for j in members))
        classes.append({"class": name, "jobs": len(members), "cones": n, "batched_ms": cbt, "plain_per_job_ms": cpt,
                        "batched_value": n / (cbt * 1e-3), "plain_value": n / (cpt * 1e-3), "speedup": cpt / cbt})
    for s_ in sc:
        s_.close()
    bt, pt = float(np.mean(batched_ms)), float(np.mean(plain_ms))
    return {"workload": f"{len(jobs)} jobs: displaced-icosphere fields of 10k-2M triangles (log-uniform), 1-16 rect "
                        "and disk lights, 4k-1M primary hits (log-uniform)",
            "jobs": len(jobs), "triangles": int(sum(w.ntris for w in jobs)),
            "points": int(sum(r.shape[0] for r in rec)), "cones_per_step": total,
            "value": total / (bt * 1e-3), "unit": UNIT, "ms_per_step": bt, "steps": steps,
            "plain_per_job": {"value": total / (pt * 1e-3), "ms_per_step": pt,
                              "path": "cc_visibility with device pointers, once per job, same stream"},
            "speedup_vs_plain_per_job": pt / bt,
            "by_job_size": classes,
            "tuned": {"points_per_warp": best.points_per_warp, "blocks_per_sm": best.blocks_per_sm,
                      "walk_order": "given" if best.flags & _lib.CC_KEEP_ORDER else "morton",
                      "graph_replay": bool(best.flags & _lib.CC_BATCH_GRAPH)},
            "tune_ms_per_candidate": [round(float(x), 3) for x in tune_ms],
            "tune_sample": "every 16th point of every job",
            "l2": "flushed between timed steps (256 MB write)", "accuracy": acc}


def served_leg(args, kernel) -> dict:
    """The serving workload: 8 resident scenes, requests of 1-8 moved or
    recoloured lights over seeded camera poses, Poisson arrivals at each rate.
    A client thread submits each request at its arrival time with pinned host
    buffers; latency is submission to results in the host buffers. Beside it,
    the plain per-request path (cc_visibility with host buffers, one request
    at a time, first come first served) under the same arrivals, from each
    request's measured time alone."""
    import threading

    import torch

    from continuum_b200 import Server, scenes

    pool = scenes.served_scenes(seed=4)
    sc = [kernel.scene(p.meshes) for p in pool]
    poses = [[torch.from_numpy(r).pin_memory() for r in p.poses] for p in pool]
    reqs = scenes.served_requests(pool, args.serve_requests, seed=5)
    cones = [poses[si][pi].shape[0] * l.shape[0] for si, pi, l in reqs]
    pts = [poses[si][pi].shape[0] for si, pi, _ in reqs]
    outs = []
    for (si, pi, l), c in zip(reqs, cones):
        P, L = poses[si][pi].shape[0], l.shape[0]
        outs.append({"full": torch.empty((L, P), dtype=torch.int64).pin_memory().numpy(),
                     "any": torch.empty((L, P), dtype=torch.int64).pin_memory().numpy(),
                     "irradiance": torch.empty((L, P), dtype=torch.float32).pin_memory().numpy(),
                     "fraction": torch.empty((L, P), dtype=torch.float32).pin_memory().numpy()})

    # The plain per-request path: each request alone through cc_visibility.
    for si, pi, l in reqs[:2]:
        kernel.visibility(sc[si], poses[si][pi].numpy(), l)
    service = []
    for (si, pi, l), o in zip(reqs, outs):
        t0 = time.perf_counter()
        kernel.visibility(sc[si], poses[si][pi].numpy(), l)
        service.append(time.perf_counter() - t0)
    service_alone = service

    def pct(x, q):
        return float(np.percentile(np.asarray(x) * 1e3, q)) if len(x) else None

    # Warm-up (untimed): one server through the first requests, so that the
    # process's first server pays no one-time costs inside a timed rate.
    srv = Server(kernel, hbm_budget=args.serve_budget_gib << 30, max_inflight=4)
    ids = [srv.add_scene(s_) for s_ in sc]
    for t in [srv.submit(ids[si], poses[si][pi].numpy(), l, o, cache_key=1 + si * 16 + pi)
              for (si, pi, l), o in list(zip(reqs, outs))[:8]]:
        srv.wait(t)
    srv.close()

    rates = [float(r) for r in args.serve_rates.split(",")]
    results = []
    for ri, rate in enumerate(rates):
        rng = np.random.default_rng(100 + ri)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
        arrivals -= arrivals[0]
        # Plain, first come first served: each request waits for the previous.
        done_at, lat_plain = 0.0, []
        for a, s_ in zip(arrivals, service_alone):
            done_at = max(done_at, a) + s_
            lat_plain.append(done_at - a)
        plain_span = done_at

        def serve(deadline_ns_per_cone):
            srv = Server(kernel, hbm_budget=args.serve_budget_gib << 30, max_inflight=4,
                         deadline_ns_per_cone=deadline_ns_per_cone)
            ids = [srv.add_scene(s_) for s_ in sc]
            tickets = [None] * len(reqs)
            refused = [False] * len(reqs)

            def client():
                t0 = time.perf_counter()
                for i, ((si, pi, l), o) in enumerate(zip(reqs, outs)):
                    wait = arrivals[i] - (time.perf_counter() - t0)
                    if wait > 0:
                        time.sleep(wait)
                    try:
                        tickets[i] = srv.submit(ids[si], poses[si][pi].numpy(), l, o, cache_key=1 + si * 16 + pi)
                    except Exception:
                        refused[i] = True

            t_start = time.perf_counter()
            th = threading.Thread(target=client)
            th.start()
            th.join()
            stats = []
            for t in tickets:
                if t is not None:
                    stats.append(srv.wait(t))
            span = time.perf_counter() - t_start
            st = srv.stats()
            srv.close()
            return tickets, refused, stats, span, st

        def small_p50(tickets, stats):
            small = [x["total_ms"] / 1e3 for x, p in zip(stats, [p for p, t in zip(pts, tickets) if t is not None])
                     if p < 100_000]
            return pct(small, 50) if small else None

        arrival = None
        if rate * float(np.mean(service_alone)) > 1.0:
            # Over capacity, where the order matters: the same arrivals again,
            # admitted in arrival order, beside the default deadline order.
            a_tickets, _, a_stats, a_span, _ = serve(0)
            a_lat = [x["total_ms"] / 1e3 for x in a_stats]
            arrival = {"deadline_ns_per_cone": 0,
                       "queries_per_s": sum(c for c, t in zip(cones, a_tickets) if t is not None) / a_span,
                       "p50_ms": pct(a_lat, 50), "p99_ms": pct(a_lat, 99),
                       "p50_ms_requests_under_100k_points": small_p50(a_tickets, a_stats)}
        tickets, refused, stats, span, st = serve(12)
        lat = [x["total_ms"] / 1e3 for x in stats]
        served_service = [(x["total_ms"] - x["queued_ms"]) / 1e3 for x in stats]
        big = [x["total_ms"] / 1e3 for x, p in zip(stats, [p for p, t in zip(pts, tickets) if t is not None])
               if p >= 1_000_000]
        big_service = [(x["total_ms"] - x["queued_ms"]) / 1e3
                       for x, p in zip(stats, [p for p, t in zip(pts, tickets) if t is not None]) if p >= 1_000_000]
        served_cones = sum(c for c, t in zip(cones, tickets) if t is not None)
        done = [i for i, t in enumerate(tickets) if t is not None]
        slowest = sorted(zip(done, stats), key=lambda x: -x[1]["total_ms"])[:3]
        results.append({
            "rate_req_s": rate, "requests": len(reqs), "completed": len(stats), "refused": int(sum(refused)),
            "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
            "p99_ms_requests_of_1M_points_or_more": pct(big, 99) if big else None,
            "p50_ms_requests_under_100k_points": small_p50(tickets, stats),
            "p50_ms_requests_of_1M_points_or_more": pct(big, 50) if big else None,
            "service_p50_ms": pct(served_service, 50), "service_p99_ms": pct(served_service, 99),
            "service_p99_ms_requests_of_1M_points_or_more": pct(big_service, 99) if big_service else None,
            "offered_load": rate * float(np.mean(service_alone)) if service_alone else None,
            "queries_per_s": served_cones / span, "requests_per_s": len(stats) / span,
            "launches": st["launches"], "lights_from_cache": st["cached_lights"], "lights_traced": st["traced_lights"],
            "peak_device_bytes": st["peak_bytes"],
            "slowest": [{"request": i, "submitted_s": round(float(arrivals[i]), 3), "points": pts[i],
                         "lights": int(reqs[i][2].shape[0]), "cached_lights": x["cached_lights"],
                         "queued_ms": round(x["queued_ms"], 1), "total_ms": round(x["total_ms"], 1),
                         "alone_ms": round(1e3 * service_alone[i], 1), "launch_requests": x["launch_requests"]}
                        for i, x in slowest],
            "admission": "earliest deadline first, 12 ns per cone",
            "arrival_order": arrival,
            "plain_per_request": {"p50_ms": pct(lat_plain, 50), "p99_ms": pct(lat_plain, 99),
                                  "queries_per_s": sum(cones) / plain_span},
        })
    acc = None
    if not args.no_accuracy:
        # Untimed: every 6th request's served results (from the last rate; a
        # strided sample of its cones) against the oracle and the plain path.
        import torch

        from oracle.oracle import OracleScene
        from oracle.parity import check_against

        dev = torch.device("cuda", torch.cuda.current_device())
        stream = torch.cuda.current_stream(dev)
        oscenes, reports, same = {}, [], True
        for i in range(0, len(reqs), 6):
            si, pi, l = reqs[i]
            if si not in oscenes:
                oscenes[si] = OracleScene(pool[si].meshes)
            recv = poses[si][pi].numpy()
            C = recv.shape[0] * l.shape[0]
            ids = strided_ids(C, args.accuracy_cones // 8)
            gpu = {k: np.asarray(outs[i][k]).reshape(-1)[ids.astype(np.int64)] for k in
                   ("full", "any", "irradiance", "fraction")}
            gpu["full"], gpu["any"] = gpu["full"].view(np.uint64), gpu["any"].view(np.uint64)
            alone = solve_on_device(kernel, sc[si], torch.from_numpy(recv).to(dev), torch.from_numpy(l).to(dev), dev,
                                    stream)
            solo = host_results(alone, ids)
            same = same and all(same_bits(gpu[k], solo[k]).all() for k in gpu)
            reports.append(check_against(oscenes[si], recv, l, gpu, partial_rows(alone["partial"], ids), cone_ids=ids,
                                         threads=cpu_threads()))
            del alone
        for o_ in oscenes.values():
            o_.close()
        acc = merge_reports(reports, f"every 6th request ({len(reports)}) of the last rate, at most "
                                     f"{args.accuracy_cones // 8} strided cones each")
        acc["served_equals_plain"] = bool(same)
    for s_ in sc:
        s_.close()
    return {"accuracy": acc,
            "workload": "8 resident displaced-icosphere scenes (50k-3M triangles, log-uniform), 3 seeded camera poses "
                        "each (16k-2M primary hits, log-uniform); requests of 1-8 lights, each a base light recoloured "
                        "or a moved light (1:1)",
            "scene_triangles": [p.ntris for p in pool], "requests_per_rate": len(reqs),
            "mean_cones_per_request": float(np.mean(cones)),
            "server": {"hbm_budget_gib": args.serve_budget_gib, "max_inflight": 4,
                       "cache_key": "scene and camera pose (recoloured lights are served from the lighting cache)"},
            "plain_per_request_path": "cc_visibility with pinned host buffers, one request at a time; latency under "
                                      "the same arrivals from each request's measured time alone, first come first served",
            "latency_terms": "total: submission to results in the host buffers; service: admission to results; "
                             "offered_load: arrival rate x mean time of a request alone (above 1: over capacity)",
            "requests_of_1M_points_or_more": int(sum(1 for p in pts if p >= 1_000_000)),
            "kernel_rate_for_16ms_at_1M_points": {
                "cones_per_s_needed_per_light": 1_000_000 / 0.016,
                "note": "a 1M-point request with L lights is L M cones: 16 ms needs 62.5 M x L cones/s"},
            "rates": results}


def instanced_leg(args, kernel, dev, stream, flush) -> dict:
    """The instanced large world: 10 displaced UV-sphere boulders (10,240
    triangles each) placed as 1,000,000 instances (10.24 billion instanced
    triangles) on a ground quad, 8 lights, 1280x720 primary hits. A full solve
    (device-timed, L2 flushed), then frames in which 1% of the instances (a
    fixed movable set) move: each frame's move (host subtree rebuild and
    upload), stale-cone marking and incremental recompute, wall-clock timed
    as one update of the cached results, after one untimed frame. The stale
    cones are recomputed through the batched form (an update job,
    cc_batch_add_update, replayed from its captured graph); the plain update
    (cc_visibility_update) recomputes a second copy of the cache beside it,
    device-timed, and the two copies must be equal."""
    import torch

    from continuum_b200 import scenes

    w = scenes.instanced_world(seed=5, n_instances=args.instances)
    n_obj = len(w.instances)
    movable = np.arange(0, n_obj - 1, 100, dtype=np.uint32)  # 1%, the ground stays
    scene = kernel.scene_instanced(w.geometries, w.instances, movable)
    rec = torch.from_numpy(w.receivers).to(dev)
    lig = torch.from_numpy(w.lights).to(dev)
    P, L = rec.shape[0], lig.shape[0]
    C = P * L
    cache = {"full": torch.empty(C, dtype=torch.int64, device=dev), "any": torch.empty(C, dtype=torch.int64, device=dev),
             "irradiance": torch.empty(C, device=dev), "fraction": torch.empty(C, device=dev)}
    ptrs = {k: v.data_ptr() for k, v in cache.items()}

    def full():
        kernel.visibility_device(scene, rec.data_ptr(), P, lig.data_ptr(), L, ptrs, stream=stream.cuda_stream)

    steps = max(1, min(args.steps, 2))
    full_ms = float(np.mean(timed_steps(torch, dev, stream, flush, full, 1, steps)))
    acc = {}
    oscene = None
    ids = strided_ids(C, args.accuracy_cones)

    def check(label):
        """Untimed: the cached results (a strided sample) against the oracle
        and against a fresh plain solve of the scene as it now is."""
        from oracle.parity import check_against

        from continuum_b200 import _lib

        gpu = host_results(cache, ids)
        fresh = solve_on_device(kernel, scene, rec, lig, dev, stream, work=True)
        solo = host_results(fresh, ids)
        capped = (fresh["work"][:, 3].cpu().numpy()[ids.astype(np.int64)] & _lib.CC_CONE_CAPPED) != 0
        differ = np.zeros(len(ids), bool)
        for k in gpu:
            differ |= ~same_bits(gpu[k], solo[k])
        rep = check_against(oscene, w.receivers, w.lights, solo, partial_rows(fresh["partial"], ids), cone_ids=ids,
                            threads=cpu_threads(), sample=f"{len(ids)} strided cones of {C}")
        rep["cache_vs_full_solve"] = {"differing_cones": int(differ.sum()), "differing_uncapped": int((differ & ~capped).sum()),
                                      "capped": int(capped.sum())}
        acc[label] = rep

    if not args.no_accuracy:
        from oracle.oracle import OracleScene

        oscene = OracleScene.instanced(w.geometries, w.instances, movable)
        check("full_solve")
    from continuum_b200 import Batch

    stale = torch.empty(C, dtype=torch.uint8, device=dev)
    plain_cache = {k: v.clone() for k, v in cache.items()}
    plain_ptrs = {k: v.data_ptr() for k, v in plain_cache.items()}
    batch = Batch(kernel)
    batch.add_update(scene, rec.data_ptr(), P, lig.data_ptr(), L, stale.data_ptr(), ptrs)
    frames = []
    # Frame 0 untimed (first-call costs and the batch's graph capture), then
    # the timed frames.
    for f in range(0, args.frames + 1):
        pl = scenes.moved_placements(w, movable, f)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        boxes = scene.move(pl)
        count = kernel.stale_cones(scene, rec.data_ptr(), P, w.lights, boxes, stale.data_ptr(),
                                   stream=stream.cuda_stream)
        e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        e0.record(stream)
        batch.submit(stream=stream.cuda_stream)
        e1.record(stream)
        batch.wait()
        ms = (time.perf_counter() - t0) * 1e3
        e2.record(stream)
        solved = kernel.visibility_update(scene, rec.data_ptr(), P, lig.data_ptr(), L, stale.data_ptr(), plain_ptrs,
                                          stream=stream.cuda_stream)
        e3.record(stream)
        torch.cuda.synchronize(dev)
        if f > 0:
            frames.append({"ms": ms, "stale_cones": count, "recomputed": solved, "stale_share": count / C,
                           "batched_recompute_ms": e0.elapsed_time(e1), "plain_update_ms": e2.elapsed_time(e3)})
        last_placements = pl
    batched_equals_plain = all(torch.equal(cache[k], plain_cache[k]) for k in cache)
    batch.close()
    del plain_cache
    if oscene is not None:
        oscene.move(last_placements)
        check(f"after_{args.frames + 1}_moving_frames")
        oscene.close()
    scene.close()
    upd = float(np.mean([fr["ms"] for fr in frames])) if frames else None
    mean = lambda key: float(np.mean([fr[key] for fr in frames])) if frames else None
    return {"workload": f"{n_obj - 1} boulder instances (10 displaced UV spheres, 10,240 triangles each) on a ground "
                        f"quad, {L} lights, 1280x720 primary hits; 1% of the instances move per frame",
            "instanced_triangles": w.instanced_tris, "points": P, "cones": C, "accuracy": acc or None,
            "full_solve": {"value": C / (full_ms * 1e-3), "unit": UNIT, "ms": full_ms, "steps": steps,
                           "timing": "CUDA events, L2 flushed"},
            "frames": frames,
            "update": {"ms_per_frame": upd, "cones_per_s_served": (C / (upd * 1e-3)) if upd else None,
                       "timing": "wall clock: host move of the movers' subtree and upload, stale-cone marking, "
                                 "recompute of the stale cones through the batched form (an update job, graph "
                                 "replay)",
                       "speedup_vs_full_solve": (full_ms / upd) if upd else None,
                       "batched_recompute_ms": mean("batched_recompute_ms"),
                       "plain_update_ms": mean("plain_update_ms"),
                       "batched_equals_plain_update": batched_equals_plain}}


def bake_leg(args, kernel, scene, w) -> dict:
    """The lighting cache's bake over the plain workload's view: pages of 8 x 8
    texels (stored 9 x 9) over the camera's 1280 x 720 hit grid (a stand-in
    for the cache's charts: one page per 8 x 8 pixels), 4 lights, nearest the
    image centre first. With a fixed budget of `--bake-budget` cones a frame
    the view warms in a few frames: device cones/s from the bake's CUDA events,
    wall time per frame with planning and staging. Then with a 14 ms frame
    target and 4 ms of camera passes: the budget the bake model settles on,
    and the bake time it gives."""
    from continuum_b200 import LightingCache, scenes
    from continuum_b200.kernel import prepare_requests

    width, height = 1280, 720
    rec, hit = scene.primary_hits(w.camera, width, height)
    pages = scenes.grid_pages(rec.reshape(height, width, 8), hit.reshape(height, width).astype(bool))
    for p in pages:
        _, py, px = p.key
        p.priority = int(abs(py * 8 + 4 - height / 2) + abs(px * 8 + 4 - width / 2))
    prepared = prepare_requests(pages)
    out = {"workload": f"{len(pages)} pages over the {width}x{height} hit grid of the plain workload, "
                       f"{w.lights.shape[0]} lights, visible fraction (light_ratio)", "pages": len(pages)}

    def run(frames_max, **opt):
        cache = LightingCache(kernel, scene, w.lights, pages=16384, **opt)
        rows, jobs_prev = [], 0
        for f in range(frames_max):
            t0 = time.perf_counter()
            st = cache.frame(prepared, period_ms=16.0, render_ms=4.0)
            rows.append({"frame": f, "budget": st["budget"], "pages": st["pages_planned"], "cones": st["jobs"],
                         "host_ms": (time.perf_counter() - t0) * 1e3, "prev_bake_ms": st["last_bake_ms"]})
            if st["pages_planned"] == 0:
                break
        cache.frame(prepared)  # reads the last bake's time
        last = cache.frame(prepared)
        for i in range(len(rows) - 1):
            rows[i]["bake_ms"] = rows[i + 1]["prev_bake_ms"]
        rows[-1]["bake_ms"] = last["last_bake_ms"] if rows[-1]["cones"] else 0.0
        resident = last["resident"]
        cache.close()
        return rows, resident

    run(2, bake_budget=args.bake_budget)  # warm-up (untimed): first use of the bake's kernels and buffers
    rows, resident = run(200, bake_budget=args.bake_budget)
    baked = [r for r in rows if r["cones"]]
    cones = sum(r["cones"] for r in baked)
    dev_ms = sum(r["bake_ms"] for r in baked)
    out["fixed_budget"] = {"bake_budget": args.bake_budget, "frames_to_warm": len(baked), "resident": resident,
                           "cones": cones, "value": cones / (dev_ms * 1e-3) if dev_ms > 0 else None, "unit": UNIT,
                           "bake_ms_per_frame": [round(r["bake_ms"], 3) for r in baked],
                           "host_ms_per_frame": [round(r["host_ms"], 3) for r in baked],
                           "timing": "CUDA events around each bake (texel upload, visibility, pool scatter)"}
    rows, resident = run(60, bake_budget=1 << 22, frame_target_ms=14.0)
    out["adaptive"] = {"frame_target_ms": 14.0, "render_ms": 4.0,
                       "budget": [round(r["budget"]) for r in rows if r["cones"]],
                       "bake_ms": [round(r["bake_ms"], 3) for r in rows if r["cones"]],
                       "frames_to_warm": sum(1 for r in rows if r["cones"])}
    return out


def sky_leg(args, kernel, dev, stream, flush, prefiltered_scene) -> dict:
    """Sky cones on the small plain workload (the ground and 64 boxes, 770
    triangles; its 256 x 256 receivers lifted 1e-4 off the ground): six
    cube-face cones per receiver (393,216 cones), the irradiance per unit
    uniform sky radiance per receiver, device-timed with CUDA events (L2
    flushed between steps). Exact sky cones reach 1e7 past each receiver over
    a 90-degree face, so their cost grows with the whole scene in view; the
    reference prefilters them, as the second measurement does on the plain
    workload at scale."""
    import torch

    from continuum_b200 import scenes

    w = scenes.box_field()
    rec_h = w.receivers.copy()
    rec_h[:, 1] = 1e-4
    scene = kernel.scene(w.meshes)
    P = rec_h.shape[0]
    rec = torch.from_numpy(rec_h).to(dev)
    out = torch.empty(P, device=dev)
    faces = torch.empty(6 * P, device=dev)

    def step():
        kernel.sky_visibility_device(scene, rec.data_ptr(), P, out.data_ptr(), faces={"irradiance": faces.data_ptr()},
                                     stream=stream.cuda_stream)

    steps = max(1, min(args.steps, 5))
    ms = float(np.mean(timed_steps(torch, dev, stream, flush, step, 2, steps)))
    mean = float(out.mean().item())
    scene.close()
    exact = {"workload": f"sky cones: 6 cube faces x {P} receivers of the small plain workload (770 triangles)",
             "cones": 6 * P, "value": 6 * P / (ms * 1e-3), "unit": UNIT, "ms": ms, "steps": steps,
             "mean_irradiance_per_unit_sky": mean, "timing": "CUDA events, L2 flushed"}
    # Prefiltered (1 bin, the reference renderer's default) on the plain
    # workload at scale: 6 faces x 921,600 primary hits over 3.07 M triangles.
    big_scene, big = prefiltered_scene
    P2 = big.receivers.shape[0]
    rec2 = torch.from_numpy(big.receivers).to(dev)
    out2 = torch.empty(P2, device=dev)
    faces2 = torch.empty(6 * P2, device=dev)
    kernel.prefilter = 1.0

    def step2():
        kernel.sky_visibility_device(big_scene, rec2.data_ptr(), P2, out2.data_ptr(),
                                     faces={"irradiance": faces2.data_ptr()}, stream=stream.cuda_stream)

    try:
        ms2 = float(np.mean(timed_steps(torch, dev, stream, flush, step2, 1, steps)))
    finally:
        kernel.prefilter = 0.0
    pre = {"workload": f"prefiltered sky cones (1 bin): 6 cube faces x {P2} primary hits of the plain workload at "
                       "scale (3.07 M triangles)", "cones": 6 * P2, "value": 6 * P2 / (ms2 * 1e-3), "unit": UNIT,
           "ms": ms2, "steps": steps, "mean_irradiance_per_unit_sky": float(out2.mean().item()),
           "timing": "CUDA events, L2 flushed"}
    return {"exact": exact, "prefiltered": pre}


def reference_arm(args, rank: int) -> None:
    """The reference's algorithm on the host cores: the oracle's FP32
    restatement of the reference's light-cone path on every host thread, each
    step a bounded strided sample of the workload's cones. Nothing of this
    library is loaded (the receivers come from the oracle's camera pass)."""
    if rank != 0:
        return
    from oracle.oracle import OracleScene

    w = workload(caster="oracle")
    oscene = OracleScene(w.meshes)
    rates = []
    total_cones, total_time = 0, 0.0
    threads = cpu_threads()
    for step in range(args.warmup + args.steps):
        rate, n, threads, dt = cpu_sample(w, target_seconds=args.reference_seconds, offset=step, oscene=oscene)
        if step >= args.warmup:
            rates.append(rate)
            total_cones += n
            total_time += dt
    value = total_cones / total_time
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_time / max(args.steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "impl": "reference",
        "config": config(1, w),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "cpu_model": cpu_model(),
                         "sample": f"{total_cones} cones in {args.steps} strided samples of the workload's "
                                   f"{w.receivers.shape[0] * w.lights.shape[0]}; the reference (Rust/WGSL) "
                                   "cannot be built here, its FP32 restatement (oracle/) runs on all host threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "inputs": "receivers from the oracle's camera pass (no library loaded)",
    }
    if not args.no_cpu_path:
        # The reference's CPU path (rect lights only) on the same workload:
        # slower than the restatement of its GPU path timed above.
        line["cpu_path"] = cpu_path_baseline(w, oscene, [i for i in range(w.lights.shape[0]) if w.lights[i][3] < 1.5],
                                             max_points=args.cpu_path_points)
    oscene.close()
    print(json.dumps(line), flush=True)


def cuda_arm(args, rank: int, world: int, local_rank: int) -> None:
    import torch

    from continuum_b200 import MaskConeKernel
    from continuum_b200.kernel import kernel_times

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = workload(args.points)
    P, L = w.receivers.shape[0], w.lights.shape[0]
    C = P * L
    kernel = MaskConeKernel(local_rank)
    scene = kernel.scene(w.meshes)
    rec = torch.from_numpy(w.receivers).to(dev)
    lig = torch.from_numpy(w.lights).to(dev)
    outs = {"full": torch.empty(C, dtype=torch.int64, device=dev), "any": torch.empty(C, dtype=torch.int64, device=dev),
            "irradiance": torch.empty(C, device=dev), "fraction": torch.empty(C, device=dev)}
    ptrs = {k: v.data_ptr() for k, v in outs.items()}
    # A dedicated stream for every timed launch (torch's default stream has
    # handle 0, which the library reads as "the context's own stream").
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        kernel.visibility_device(scene, rec.data_ptr(), P, lig.data_ptr(), L, ptrs, stream=stream.cuda_stream)

    # This library's kernels per step: morton_keys (Morton walk order, when
    # there are more than 64 points), light_order_kernel (two lights or
    # more), and per split chunk the cone setup, the packet pass, the solo
    # pass and the integration.
    morton = P > 64
    chunks = (C + (1 << 25) - 1) >> 25
    launches_per_step = 4 * chunks + (1 if morton else 0) + (1 if L >= 2 else 0)

    # Work counters (an untimed counted run): the algorithmic bytes per cone.
    work = torch.empty(C, 4, dtype=torch.int32, device=dev)
    kernel.visibility_device(scene, rec.data_ptr(), P, lig.data_ptr(), L, {**ptrs, "work": work.data_ptr()},
                             stream=stream.cuda_stream)
    torch.cuda.synchronize(dev)
    wk = work.cpu().numpy().view(np.uint32)
    n_obj, n_blas, n_tri = (float(wk[:, i].astype(np.float64).sum()) for i in range(3))
    status = wk[:, 3]
    algo_bytes = C * (32 + 16 + 24) + NODE_BYTES * (n_obj + n_blas) + TRI_BYTES * n_tri
    del work
    kernel_times(kernel)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    kernel_times(kernel)

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize(dev)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with Clocks(local_rank) as clk:
        for i in range(args.steps):
            flush.zero_()
            starts[i].record(stream)
            step()
            ends[i].record(stream)
        torch.cuda.synchronize(dev)
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    kt = kernel_times(kernel)
    elapsed = max_over_ranks(float(sum(step_ms)) / 1e3, world, dev)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    value = replica_value(C, args.steps, world, elapsed)
    packet_ms = float(np.mean(kt[:, 0])) if len(kt) else None
    solo_ms = float(np.mean(kt[:, 1])) if len(kt) else None

    # End to end through the C ABI with host buffers (pinned), copies included.
    rec_h = torch.from_numpy(w.receivers).pin_memory().numpy()
    lig_h = np.ascontiguousarray(w.lights)
    e2e_steps = max(1, min(args.steps, 5))
    host_out = {k: torch.empty(C, dtype=dt).pin_memory().numpy() for k, dt in
                (("full", torch.int64), ("any", torch.int64), ("irradiance", torch.float32), ("fraction", torch.float32))}
    from continuum_b200 import _lib
    import ctypes as Cc

    opt = kernel.options()
    o = _lib.Outputs(host_out["full"].ctypes.data, host_out["any"].ctypes.data, None,
                     host_out["irradiance"].ctypes.data, host_out["fraction"].ctypes.data, None)

    def e2e_step():
        _lib.check(_lib.load().cc_visibility(kernel.handle, scene.handle, rec_h.ctypes.data, P, lig_h.ctypes.data, L,
                                             Cc.byref(opt), Cc.byref(o), None))

    if not args.no_e2e:
        e2e_step()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(0 if args.no_e2e else e2e_steps):
        e2e_step()
    e2e_time = max_over_ranks(max(time.perf_counter() - t0, 1e-9), world, dev)
    e2e_value = replica_value(C, e2e_steps, world, e2e_time)
    kernel_times(kernel)

    if rank != 0:
        scene.close()
        kernel.close()
        return

    from continuum_b200 import _lib as L_
    peaks_path = ROOT / "MEASURED_PEAKS.json"
    peak, peak_src = 6650.0, "fallback"
    if peaks_path.exists():
        try:
            peak, peak_src = float(json.loads(peaks_path.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    achieved = algo_bytes / (packet_ms * 1e-3) / 1e9 if packet_ms else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded)", "impl": "cuda", "config": config(world, w),
        "e2e": None if args.no_e2e else {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(rec_h.nbytes + lig_h.nbytes),
                "d2h_bytes_per_step": int(sum(v.nbytes for v in host_out.values()) + 8),
                "steps": e2e_steps, "path": "cc_visibility with host buffers (pinned), scene resident"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     # DRAM bytes of one packet-pass launch of this workload at
                     # full size (dram__bytes_read.sum + dram__bytes_write.sum),
                     # from the ncu capture committed under profiles/, not from
                     # this run; null for other sizes.
                     "traffic": PACKET_PASS_DRAM_BYTES if C == FULL_CONES else None,
                     "traffic_source": "ncu capture of the packet pass at full size (profiles/), not this run",
                     "peak_source": peak_src,
                     "kernel": "visibility_kernel (packet pass)", "kernel_ms": packet_ms,
                     "solo_pass_and_integration_ms": solo_ms,
                     "algorithmic_bytes_per_launch": algo_bytes,
                     "bytes_model": "per cone: 32 B receiver + 16 B light + 24 B outputs + 48 B x (object + "
                                    "triangle-hierarchy nodes tested) + 48 B x triangles tested",
                     "work_per_cone": {"object_nodes": n_obj / C, "triangle_nodes": n_blas / C,
                                       "triangles": n_tri / C},
                     "note": "most node and triangle reads hit L1/L2; the kernel is issue-bound, see profiles/"},
        "gpu_launches": launches_per_step * args.steps,
        "library_launches": {"cub_radix_sort": 6 * args.steps if morton else 0},
        "clocks": clk.summary(),
        "status": {"capped": int(((status & L_.CC_CONE_CAPPED) != 0).sum()),
                   "rewalked": int(((status & L_.CC_CONE_REWALKED) != 0).sum()),
                   "diverged": int(((status & L_.CC_CONE_DIVERGED) != 0).sum())},
    }
    forms = set(args.forms.split(",")) if args.forms else set()

    def settle():
        """Frees what the previous leg left (its tensors and pinned host
        buffers, held by Python's collector and torch's caches) before the
        next leg, so that no deferred free lands in a timed region."""
        import gc

        gc.collect()
        torch.cuda.synchronize(dev)
        torch.cuda.empty_cache()
        host_empty = getattr(torch._C, "_host_emptyCache", None)
        if host_empty is not None:
            host_empty()

    oscene = None
    if world == 1 and not (args.no_accuracy and args.no_cpu_baseline and args.no_cpu_path):
        from oracle.oracle import OracleScene

        oscene = OracleScene(w.meshes)
    if world == 1 and not args.no_accuracy:
        # Untimed: every cone of the step against the oracle (FP32 bar, FP64 error).
        settle()
        line["accuracy"] = {"plain_at_scale": plain_accuracy(kernel, scene, oscene, w.receivers, w.lights, dev, stream)}
    if "small" in forms:
        settle()
        line["small"] = small_leg(args, kernel, dev, stream, flush)
        if line["small"].get("accuracy") is not None:
            line.setdefault("accuracy", {})["small"] = line["small"]["accuracy"]
    if "batched" in forms:
        settle()
        line["batched"] = batched_leg(args, kernel, dev, stream, flush)
    if "served" in forms:
        settle()
        line["served"] = served_leg(args, kernel)
    if "instanced" in forms:
        settle()
        line["instanced"] = instanced_leg(args, kernel, dev, stream, flush)
    if "bake" in forms:
        settle()
        line["bake"] = bake_leg(args, kernel, scene, w)
    if "sky" in forms:
        settle()
        line["sky"] = sky_leg(args, kernel, dev, stream, flush, (scene, w))
    for form in ("batched", "served"):
        if line.get(form, {}).get("accuracy") is not None:
            line.setdefault("accuracy", {})[form] = line[form]["accuracy"]
    if line.get("instanced", {}).get("accuracy") is not None:
        line.setdefault("accuracy", {})["instanced"] = line["instanced"]["accuracy"]
    if world == 1 and not args.no_cpu_baseline:
        rate, n, threads, dt = cpu_sample(w, target_seconds=args.cpu_seconds, oscene=oscene)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "cpu_model": cpu_model(),
                                "sample": f"{n} strided cones of {C} ({dt:.1f} s wall); FP32 restatement "
                                          "of the reference's GPU path (oracle/) on every host thread"}
        if not args.no_cpu_path:
            line["cpu_baseline"]["cpu_path"] = cpu_path_baseline(
                w, oscene, [i for i in range(L) if w.lights[i][3] < 1.5], max_points=args.cpu_path_points)
    if oscene is not None:
        oscene.close()
    print(json.dumps(line), flush=True)
    scene.close()
    kernel.close()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=1.5)
    ap.add_argument("--reference-seconds", type=float, default=2.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cpu-path", action="store_true", help="skip the reference CPU path's 1- and all-thread timings")
    ap.add_argument("--cpu-path-points", type=int, default=8192,
                    help="receivers per rect light of the plain-at-scale workload's CPU-path sample")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the untimed accuracy report (profiling runs)")
    ap.add_argument("--accuracy-cones", type=int, default=65536,
                    help="cones checked per sampled form (batched and served: an eighth per job or request)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--forms", default="small,batched,served,instanced,bake,sky",
                    help="workloads and forms measured beside the plain line (comma list of small, batched, served, "
                         "instanced, bake, sky; none)")
    ap.add_argument("--bake-budget", type=int, default=1 << 20, help="cones a frame of the bake leg's fixed budget")
    ap.add_argument("--instances", type=int, default=1_000_000)
    ap.add_argument("--frames", type=int, default=3, help="moving frames of the instanced leg")
    ap.add_argument("--batch-jobs", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=3, help="timed steps of the batched leg (at most --steps)")
    ap.add_argument("--serve-requests", type=int, default=48)
    ap.add_argument("--serve-rates", default="5,10,20,50,200,2000", help="Poisson arrival rates (requests/s)")
    ap.add_argument("--serve-budget-gib", type=int, default=16)
    ap.add_argument("--points", type=int, default=0,
                    help="keep a strided subset of this many receivers (profiling runs; not a bench line)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        cuda_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
