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


GEOM_FIELDS = ["depth", "means2D", "cov3D", "conic_opac", "rgb", "tiles", "offsets"]


def geometry_mismatches(mine: dict, orc: dict, visible=None) -> dict:
    """Bit mismatches per geometry field (float fields compared as fp32 bits).
    ``visible``: only Gaussians that passed the projection are compared for
    fields the reference leaves unwritten for culled ones."""
    out = {}
    for k in GEOM_FIELDS:
        a, b = np.asarray(mine[k]), np.asarray(orc[k])
        if b.dtype.kind == "f":
            b = b.astype(np.float32)
        if visible is not None and k not in ("cov3D", "tiles", "offsets"):
            a, b = a[visible], b[visible]
        out[k] = bit_mismatch(a, b)
    out["radii"] = bit_mismatch(mine["radii"], orc["radii"])
    if "clamped" in mine and "clamped" in orc:
        out["clamped"] = bit_mismatch(mine["clamped"], orc["clamped"])
    return out


def ncontrib_check(mine_nc, orc_nc, orc_margin, margin=1e-5):
    """Contributor counts must match except at pixels whose blend decisions
    sit within ``margin`` (relative) of an alpha or transmittance threshold,
    where the device exp and the C library's exp may round differently."""
    diff = np.asarray(mine_nc) != np.asarray(orc_nc)
    unexplained = diff & (np.asarray(orc_margin) >= margin)
    return dict(n_diff=int(diff.sum()), n_unexplained=int(unexplained.sum()), n=int(diff.size), mask=diff)


# fp32 accumulation of N terms in different orders: the results differ by at
# most a few ulps of the sum of |terms|; 64 ulps of margin.
ACC_ULPS = 64 * 2.0 ** -24


# Comparisons of this implementation with itself (batched vs single-view
# calls, the preamble folded in vs run apart, a request alone vs in a mixed
# batch, one launch shape vs another) differ only in the order of float
# atomic additions, and no oracle sums of |terms| are at hand there; they
# bound that order's effect by a fraction of the largest component of the
# same Gaussian instead, and also require norm-relative agreement <= 1e-5.
SAME_IMPL_ROW_RTOL = 1e-3


def grad_check(a, b, row_rtol=0.0, abs_sum=None) -> dict:
    """Gradient agreement of ``a`` with ``b``.  Elementwise bound
    |a-b| <= ATOL + RTOL*|b| [+ ACC_ULPS * sum|terms| when the per-element sum
    of absolute contributions is given] [+ row_rtol * max|b over the same
    Gaussian|, for comparisons of this implementation with itself]: the extra
    terms cover components that cancel to much less than their summands,
    where fp32 accumulation order dominates.  n_elem_strict counts the
    elements outside the plain ATOL + RTOL*|b| bound."""
    a = np.asarray(a, np.float64).reshape(len(a), -1)
    b = np.asarray(b, np.float64).reshape(len(b), -1)
    d = np.abs(a - b)
    row = np.abs(b).max(axis=1, keepdims=True) if b.size else b
    tol = ATOL + RTOL * np.abs(b) + row_rtol * row
    if abs_sum is not None:
        tol = tol + ACC_ULPS * np.asarray(abs_sum, np.float64).reshape(d.shape)
    nb = float(np.linalg.norm(b.ravel())) or 1.0
    return dict(norm_rel=float(np.linalg.norm((a - b).ravel()) / nb), n_bad=int((d > tol).sum()),
                n_elem_strict=int((d > ATOL + RTOL * np.abs(b)).sum()), max_abs=float(d.max()) if d.size else 0.0,
                n=int(d.size))


GRAD_NAMES = ["dL_dmeans2D", "dL_dcolors", "dL_dopacity", "dL_dmeans3D", "dL_dcov3D", "dL_dsh", "dL_dscales",
              "dL_drotations"]
