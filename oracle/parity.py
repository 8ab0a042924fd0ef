"""ORACLE — test infrastructure: comparison of CUDA results with the oracle's,
with the path's tolerances. Used by tests/ and by bench.py's untimed
accuracy report, as the checker.

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


def accuracy(gpu: dict, orc32: dict, orc64: dict | None = None, sample: str = "every cone") -> dict:
    """The accuracy report of one workload: the bar's statistics against the
    FP32 oracle (`orc32`, with `unshadowed`), and the error against the FP64
    oracle (`orc64`): the largest |fraction - fraction64|, the largest
    irradiance error relative to the cone's unshadowed light (floored as the
    bar floors it), and the share of cones whose mask words equal the FP64
    run's. `gpu` and the oracles' arrays are per cone, in the same order;
    partial coverages (where given) trace disagreeing bits. Does not assert."""
    stats = compare(gpu, orc32, orc32.get("unshadowed"), check=False)
    rec = {"cones": stats["cones"], "sample": sample, "word_agreement": stats["word_agreement"],
           "max_dfraction": stats.get("max_fraction_diff"),
           "max_dirradiance_rel": stats.get("max_irradiance_diff_rel"),
           "mismatched_cones": stats["mismatched_cones"], "untraced_bits": stats["untraced_bits"]}
    if orc64 is not None:
        n = rec["cones"]
        g_frac = np.asarray(gpu["fraction"], np.float64).reshape(-1)
        f64 = np.asarray(orc64["fraction"], np.float64).reshape(-1)
        o_frac = np.asarray(orc32["fraction"], np.float64).reshape(-1)
        err = {"fraction": float(np.abs(g_frac - f64).max()) if n else 0.0,
               "fraction_oracle_fp32": float(np.abs(o_frac - f64).max()) if n else 0.0}
        u = np.asarray(orc64["unshadowed"], np.float64).reshape(-1)
        m = u > 0
        if m.any() and gpu.get("irradiance") is not None:
            scale = np.maximum(u[m], IRRADIANCE_FLOOR * u[m].max())
            gi = np.asarray(gpu["irradiance"], np.float64).reshape(-1)[m]
            oi = np.asarray(orc32["irradiance"], np.float64).reshape(-1)[m]
            i64 = np.asarray(orc64["irradiance"], np.float64).reshape(-1)[m]
            err["irradiance_rel"] = float((np.abs(gi - i64) / scale).max())
            err["irradiance_rel_oracle_fp32"] = float((np.abs(oi - i64) / scale).max())
        g_full = np.asarray(gpu["full"]).reshape(-1)
        g_any = np.asarray(gpu["any"]).reshape(-1)
        err["word_agreement"] = float(((g_full == np.asarray(orc64["full"]).reshape(-1)) &
                                       (g_any == np.asarray(orc64["any"]).reshape(-1))).mean()) if n else 1.0
        rec["fp64_max_abs_err"] = err
    rec["meets_bar"] = bool(rec["word_agreement"] >= WORD_AGREEMENT and
                            (rec["max_dfraction"] is None or rec["max_dfraction"] <= FRACTION_TOL) and
                            (rec["max_dirradiance_rel"] is None or rec["max_dirradiance_rel"] <= IRRADIANCE_TOL) and
                            rec["untraced_bits"] == 0)
    return rec


def _words_agree(a: dict, b: dict) -> np.ndarray:
    return ((np.asarray(a["full"]).reshape(-1) == np.asarray(b["full"]).reshape(-1)) &
            (np.asarray(a["any"]).reshape(-1) == np.asarray(b["any"]).reshape(-1)))


def check_against(oscene, receivers: np.ndarray, lights: np.ndarray, gpu: dict, gpu_partial=None,
                  cone_ids: np.ndarray | None = None, fp64: bool = True, threads: int | None = None,
                  sample: str = "every cone", **options) -> dict:
    """The accuracy report of GPU results `gpu` (full, any, irradiance,
    fraction per cone, for every cone or the `cone_ids` subset, in that
    order) against the oracle scene `oscene` on the same receivers and
    lights. `gpu_partial(positions)` returns the GPU's 64 coverages of those
    positions, to trace disagreeing bits (None: not traced). `options` go to
    OracleScene.visibility.

    The oracle runs the reference's arithmetic with three summations of each
    mesh's cells (the values added are the same): the library's (each add
    rounded to 2^-24 of a bin into exact integer cells), against which the
    parity bar is held; the reference's own (f32 adds in walk order); and
    exact sums (double). The report gives the bar's statistics, the
    agreement with the reference's summation (every disagreeing bit traced),
    how far each summation's words are from exact sums, and the error
    against the FP64 oracle."""
    from .oracle import SUM_EXACT, SUM_FIXED, SUM_WALK_ORDER

    def run(**kw):
        return oscene.visibility(receivers, lights, cone_ids=cone_ids, threads=threads, partial=False,
                                 **{**options, **kw})

    fixed = run(accumulate=SUM_FIXED)
    walk = run(accumulate=SUM_WALK_ORDER)
    exact = run(accumulate=SUM_EXACT)
    o64 = run(precision=8) if fp64 else None
    rec = accuracy(gpu, fixed, o64, sample=sample)
    rec["oracle_summation"] = "the library's (fixed point, 2^-24 of a bin per add)"

    def trace(orc_kind: int, agree: np.ndarray) -> int:
        bad = np.nonzero(~agree)[0]
        if not bad.size:
            return 0
        if gpu_partial is None:
            return -1
        ids = bad.astype(np.uint64) if cone_ids is None else np.asarray(cone_ids, np.uint64)[bad]
        ob = oscene.visibility(receivers, lights, cone_ids=ids, threads=threads, partial=True,
                               **{**options, "accumulate": orc_kind})
        sub = {"full": np.asarray(gpu["full"]).reshape(-1)[bad], "any": np.asarray(gpu["any"]).reshape(-1)[bad],
               "partial": np.asarray(gpu_partial(bad)).reshape(-1, 64)}
        return compare(sub, ob, check=False)["untraced_bits"]

    a_fixed = _words_agree(gpu, fixed)
    rec["untraced_bits"] = trace(SUM_FIXED, a_fixed)
    rec["meets_bar"] = bool(rec["untraced_bits"] == 0 and rec["word_agreement"] >= WORD_AGREEMENT and
                            (rec["max_dfraction"] or 0.0) <= FRACTION_TOL and
                            (rec["max_dirradiance_rel"] or 0.0) <= IRRADIANCE_TOL)
    a_walk = _words_agree(gpu, walk)
    n = a_walk.size
    d = np.abs(np.asarray(gpu["fraction"], np.float64).reshape(-1) - np.asarray(walk["fraction"], np.float64))
    rec["reference_summation"] = {
        "word_agreement": float(a_walk.mean()) if n else 1.0, "mismatched_cones": int((~a_walk).sum()),
        "untraced_bits": trace(SUM_WALK_ORDER, a_walk),
        "max_dfraction": float(d.max()) if n else 0.0,
        "cones_dfraction_over_1e-3": int((d > FRACTION_TOL).sum()),
        "exact_sums_word_agreement": {"reference_summation": float(_words_agree(walk, exact).mean()) if n else 1.0,
                                      "library": float(_words_agree(gpu, exact).mean()) if n else 1.0},
    }
    if o64 is not None:
        d64 = np.abs(np.asarray(gpu["fraction"], np.float64).reshape(-1) - np.asarray(o64["fraction"], np.float64))
        rec["fp64_max_abs_err"]["fraction_p999"] = float(np.quantile(d64, 0.999)) if n else 0.0
        rec["fp64_max_abs_err"]["cones_dfraction_over_1e-3"] = int((d64 > FRACTION_TOL).sum())
    return rec
