"""Image comparison with the reference's formulas, in double precision
(reference src/benchmark/comparison.cpp:7-35, gate in
src/tools/compare_main.cpp:131-135)."""
from __future__ import annotations

import numpy as np

GATE_L2 = 1e-5
GATE_CORR = 0.9999


def compare_images(ref, test) -> dict:
    a = np.asarray(ref, np.float64).ravel()
    b = np.asarray(test, np.float64).ravel()
    if a.size != b.size:
        raise ValueError("image size mismatch in comparison")
    m = dict(n=int(a.size), max_abs=0.0, mean_abs=0.0, rms=0.0, l2_relative=0.0, max_relative=0.0,
             correlation=0.0, ref_max_abs=0.0, test_max_abs=0.0, argmax=0)
    if a.size == 0:
        return m
    d = a - b
    ad = np.abs(d)
    m["argmax"] = int(np.argmax(ad))
    m["max_abs"] = float(ad[m["argmax"]])
    m["mean_abs"] = float(ad.sum() / a.size)
    sum_sq = float((d * d).sum())
    ref_sq = float((a * a).sum())
    test_sq = float((b * b).sum())
    cross = float((a * b).sum())
    m["rms"] = float(np.sqrt(sum_sq / a.size))
    m["ref_max_abs"] = float(np.abs(a).max())
    m["test_max_abs"] = float(np.abs(b).max())
    m["l2_relative"] = float(np.sqrt(sum_sq / ref_sq)) if ref_sq > 0 else 0.0
    m["max_relative"] = m["max_abs"] / m["ref_max_abs"] if m["ref_max_abs"] > 0 else 0.0
    den = np.sqrt(ref_sq * test_sq)
    m["correlation"] = float(cross / den) if den > 0 else 0.0
    return m


def gate_pass(m: dict, l2: float = GATE_L2, corr: float = GATE_CORR) -> bool:
    return m["l2_relative"] < l2 and m["correlation"] > corr
