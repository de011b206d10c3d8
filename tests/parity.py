"""Comparison helpers for the parity tests.

`contraction_stats` states how far float32 results are from the oracle's
FP-contraction build (the same restatement with a*b+c contracted into FMAs,
the rounding the reference's ISPC build uses by default).  The device
rounds every operation in source order, like the oracle's parity build, so
it is compared with that build bit for bit and with the contraction build
within a stated tolerance:

    |got - want| <= 4 ULP(want)   or   |got - want| <= 1e-6 * max(|want|, 1)

(ULP counts grow without bound near zero crossings, where a lerp cancels;
the second form bounds those by the field's scale.)
"""
from __future__ import annotations

import numpy as np

ULP_BOUND = 4
REL_BOUND = 1e-6


def ordered(a):
    """float32 -> int64 keys whose differences count ULPs across zero."""
    b = np.ascontiguousarray(a, np.float32).view(np.int32).astype(np.int64)
    return np.where(b < 0, -(b & 0x7FFFFFFF), b)


def contraction_stats(got, want):
    """dict(n, nan_mismatch, max_ulp, max_rel, outside) over all elements;
    NaN must be NaN on both sides, `outside` counts elements beyond both
    bounds."""
    g = np.asarray(got, np.float32).reshape(-1)
    w = np.asarray(want, np.float32).reshape(-1)
    gn, wn = np.isnan(g), np.isnan(w)
    ok = ~(gn | wn)
    ulp = np.abs(ordered(g[ok]) - ordered(w[ok]))
    d = np.abs(g[ok].astype(np.float64) - w[ok].astype(np.float64))
    rel = d / np.maximum(np.abs(w[ok].astype(np.float64)), 1.0)
    outside = int(np.count_nonzero((ulp > ULP_BOUND) & (rel > REL_BOUND)))
    return {"n": int(g.size), "nan_mismatch": int(np.count_nonzero(gn != wn)),
            "max_ulp": int(ulp.max()) if ulp.size else 0, "max_rel": float(rel.max()) if rel.size else 0.0,
            "outside": outside}


def assert_within_contraction(got, want, what=""):
    s = contraction_stats(got, want)
    assert s["nan_mismatch"] == 0 and s["outside"] == 0, f"{what}: {s}"
    return s
