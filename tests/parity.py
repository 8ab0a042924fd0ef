"""Comparison of CUDA results with the oracle's, with the path's tolerances.

The bar (stated once, used by every parity test):
  * FULL and ANY mask words agree on at least 99.9% of cones, and every
    disagreeing bit is explained by an edge within 1e-5 of a bin boundary:
    a FULL disagreement has coverage within 2e-5 of whole on both sides, an
    ANY disagreement coverage below 2e-5 on both sides (a sliver that thin);
  * visible fractions agree within 1e-3 absolute;
  * irradiance agrees within 2e-3 of the cone's unshadowed light, floored
    at 1e-3 of the brightest cone's: near a light's horizon, or at a spot's
    edge, the unshadowed light tends to zero and f32 loses it (on these
    cases the oracle's own FP32 run differs from its FP64 run by up to
    7.3e-4 of that scale, and by up to 6x of the raw unshadowed value). The
    reference's own GPU-vs-CPU bound, 1e-4 of the light's weight
    (gpu.rs:330-336), is checked on the reference's test scenes.
"""
from __future__ import annotations

import numpy as np

WORD_AGREEMENT = 0.999
FRACTION_TOL = 1e-3
IRRADIANCE_TOL = 2e-3
IRRADIANCE_FLOOR = 1e-3
EDGE_SLACK = 2e-5


def bits(words: np.ndarray) -> np.ndarray:
    """(n,) uint64 -> (n, 64) bool, bin b = bit b."""
    w = np.ascontiguousarray(words, dtype=np.uint64).reshape(-1)
    return ((w[:, None] >> np.arange(64, dtype=np.uint64)[None, :]) & np.uint64(1)).astype(bool)


def compare(gpu: dict, orc: dict, unshadowed: np.ndarray | None = None, check: bool = True) -> dict:
    """Statistics of GPU vs oracle (flattened per cone); asserts the bar if `check`."""
    g_full = np.asarray(gpu["full"]).reshape(-1)
    g_any = np.asarray(gpu["any"]).reshape(-1)
    o_full = np.asarray(orc["full"]).reshape(-1)
    o_any = np.asarray(orc["any"]).reshape(-1)
    n = g_full.size
    agree = (g_full == o_full) & (g_any == o_any)
    stats = {"cones": int(n), "word_agreement": float(agree.mean()) if n else 1.0}
    if "fraction" in gpu and gpu["fraction"] is not None:
        d = np.abs(np.asarray(gpu["fraction"]).reshape(-1) - np.asarray(orc["fraction"]).reshape(-1))
        stats["max_fraction_diff"] = float(d.max()) if n else 0.0
    if unshadowed is not None and gpu.get("irradiance") is not None:
        u = np.asarray(unshadowed).reshape(-1)
        di = np.abs(np.asarray(gpu["irradiance"]).reshape(-1) - np.asarray(orc["irradiance"]).reshape(-1))
        m = u > 0
        if m.any():
            scale = np.maximum(u[m], IRRADIANCE_FLOOR * u[m].max())
            stats["max_irradiance_diff_rel"] = float((di[m] / scale).max())
        else:
            stats["max_irradiance_diff_rel"] = 0.0
    # Trace every disagreeing bit through the coverages on both sides.
    untraced = 0
    bad = np.nonzero(~agree)[0]
    if bad.size and gpu.get("partial") is not None and orc.get("partial") is not None:
        gp = np.asarray(gpu["partial"]).reshape(n, 64)[bad]
        op = np.asarray(orc["partial"]).reshape(n, 64)[bad]
        fb = bits(g_full[bad]) != bits(o_full[bad])
        ab = bits(g_any[bad]) != bits(o_any[bad])
        full_ok = np.minimum(gp, op) >= 1.0 - 1e-5 - EDGE_SLACK
        any_ok = np.maximum(gp, op) <= EDGE_SLACK
        untraced = int((fb & ~full_ok).sum() + (ab & ~any_ok).sum())
    elif bad.size:
        untraced = -1  # no coverages to trace with
    stats["mismatched_cones"] = int(bad.size)
    stats["untraced_bits"] = untraced
    if check:
        assert stats["word_agreement"] >= WORD_AGREEMENT, stats
        if "max_fraction_diff" in stats:
            assert stats["max_fraction_diff"] <= FRACTION_TOL, stats
        if "max_irradiance_diff_rel" in stats:
            assert stats["max_irradiance_diff_rel"] <= IRRADIANCE_TOL, stats
        assert untraced == 0, stats
    return stats


def flat(v) -> dict:
    """A Visibility (L, P, ...) as per-cone arrays in cone order."""
    out = {}
    for k in ("full", "any", "irradiance", "fraction"):
        a = getattr(v, k)
        if a is not None:
            out[k] = a.reshape(-1)
    if v.partial is not None:
        out["partial"] = v.partial.reshape(-1, 64)
    if v.work is not None:
        out["work"] = v.work.reshape(-1, 4)
    return out
