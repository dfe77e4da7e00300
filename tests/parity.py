"""Comparison helpers shared by the parity tests.

All comparisons report counts and worst errors per result so a test can both
assert and print them.  Bit-exact fields are compared as raw bits.
"""
from __future__ import annotations

import numpy as np

# Floating-point tolerance for images and gradients (fp32), elementwise:
# |a - b| <= ATOL + RTOL * |b|.
ATOL = 1e-5
RTOL = 1e-4


def bits(a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.float32:
        return a.view(np.uint32)
    if a.dtype == np.float64:
        return a.view(np.uint64)
    return a


def bit_mismatch(a, b) -> int:
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return -1
    if a.dtype != b.dtype:
        b = b.astype(a.dtype)
    return int(np.count_nonzero(bits(a) != bits(b)))


def err_stats(a, b, atol=ATOL, rtol=RTOL) -> dict:
    """Errors of ``a`` against the reference ``b``."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.abs(a - b)
    tol = atol + rtol * np.abs(b)
    bad = d > tol
    nb = float(np.linalg.norm(b.ravel())) or 1.0
    return dict(max_abs=float(d.max()) if d.size else 0.0,
                max_rel=float((d / np.maximum(np.abs(b), 1e-30)).max()) if d.size else 0.0,
                norm_rel=float(np.linalg.norm((a - b).ravel()) / nb),
                n_bad=int(bad.sum()), n=int(d.size),
                worst_excess=float((d - tol).max()) if d.size else 0.0)


def spill_classes(ref_keys, ref_vals, orc_keys, orc_vals, candidates) -> dict:
    """Classify unsorted-slot differences between the reference and the
    lowest-index-wins spill model: slots with one candidate writer must match;
    slots with several candidates may differ only where the reference's writes
    raced across warps."""
    R = min(len(ref_keys), len(orc_keys))
    diff = (ref_keys[:R] != orc_keys[:R]) | (ref_vals[:R] != orc_vals[:R])
    cand = candidates[:R]
    return dict(R=int(R), n_diff=int(diff.sum()), n_diff_single=int((diff & (cand <= 1)).sum()),
                n_multi=int((cand > 1).sum()), n_diff_multi=int((diff & (cand > 1)).sum()))
