"""Benchmark: cone-visibility queries per second on the plain-at-scale workload.

One step = one visibility solve of every (shading point, light) cone of the
plain-at-scale workload: 150 displaced icospheres (subdivision 5, 3,072,002
triangles with the ground quad), four lights (2 x 1 and 4 x 4 m rects, disks
of radius 0.5 and 1.5 m as one-sided sphere lights), and the 921,600 primary
hits of a 1280 x 720 camera: 3,686,400 cones. Synthetic, seeded data.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

The CUDA arm prints one JSON line with the device-resident throughput
(`value`), the end-to-end throughput through the C ABI with host buffers
(`e2e`), the dominant kernel's roofline, a timed CPU baseline (the oracle's
FP32 restatement of the reference's path on the host cores, a bounded
sample), the SM clocks seen during the timed region and the kernel launch
count. The reference arm times the reference's algorithm on the host cores
(the reference is Rust + WGSL and cannot be built or run here; its FP32
restatement in oracle/ stands in for it).
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


def workload(points: int = 0):
    from continuum_b200 import scenes

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


def cpu_sample(w, target_seconds: float, offset: int = 0):
    """Times the oracle (FP32, all host threads) on a strided sample of cones
    sized for about `target_seconds` of wall time. Returns (cones/s, cones, threads)."""
    from oracle.oracle import OracleScene

    threads = cpu_threads()
    scene = OracleScene(w.meshes)
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


def traffic_per_cone():
    """DRAM bytes per cone of the packet kernel from the committed ncu summary
    (profiles/visibility_kernel_icosphere_field.md), or None."""
    p = ROOT / "profiles" / "visibility_kernel_icosphere_field.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("dram_bytes_per_cone:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def reference_arm(args, rank: int) -> None:
    if rank != 0:
        return
    w = workload()
    rates = []
    total_cones, total_time = 0, 0.0
    threads = cpu_threads()
    for step in range(args.warmup + args.steps):
        rate, n, threads, dt = cpu_sample(w, target_seconds=args.reference_seconds, offset=step)
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
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{total_cones} cones in {args.steps} strided samples of the workload's "
                                   f"{w.receivers.shape[0] * w.lights.shape[0]}; the reference (Rust/WGSL) "
                                   "cannot be built here, its FP32 restatement (oracle/) runs on all host threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
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
    # there are more than 64 points), the packet pass and the solo pass.
    morton = P > 64
    launches_per_step = 2 + (1 if morton else 0)

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
    elapsed = float(sum(step_ms)) / 1e3
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([elapsed], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
        dist.barrier()
    value = world * C * args.steps / elapsed
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
    e2e_time = max(time.perf_counter() - t0, 1e-9)
    if world > 1:
        t = torch.tensor([e2e_time], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_time = float(t.item())
    e2e_value = world * C * e2e_steps / e2e_time
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
    tpc = traffic_per_cone()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded)", "impl": "cuda", "config": config(world, w),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(rec_h.nbytes + lig_h.nbytes),
                "d2h_bytes_per_step": int(sum(v.nbytes for v in host_out.values()) + 8),
                "steps": e2e_steps, "path": "cc_visibility with host buffers (pinned), scene resident"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": (tpc * C) if tpc else None, "peak_source": peak_src,
                     "kernel": "visibility_kernel (packet pass)", "kernel_ms": packet_ms, "solo_pass_ms": solo_ms,
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
    if world == 1 and not args.no_cpu_baseline:
        rate, n, threads, dt = cpu_sample(w, target_seconds=args.cpu_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{n} strided cones of {C} ({dt:.1f} s wall); FP32 restatement "
                                          "of the reference's path (oracle/)"}
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
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
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
