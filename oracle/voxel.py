"""CPU oracle for the voxel occupancy field -- TEST INFRASTRUCTURE ONLY.

A direct restatement of the reference's brute-force kernel
(``compute_voxel_field.cu:6-86``) in numpy, one voxel row at a time: every
voxel tests every Gaussian's mean against its block's grown bounds and sums
opacity * exp(power) over the Gaussians that pass, in Gaussian order.  The
voxel coordinates, block indices and bounds are evaluated in float32 as the
kernel evaluates them (``precision="f32"``, the default), or in float64
(``"f64"``); the Gaussian terms in the chosen precision.  Only the GPU tests
call it, on small grids.
"""
from __future__ import annotations

import numpy as np


def voxel_field(means, covs, opacities, resolution: int, num_blocks: int, relax_ratio: float,
                precision: str = "f32") -> np.ndarray:
    """[R, R, R] array, x fastest (occ[k, j, i])."""
    dt = np.float32 if precision == "f32" else np.float64
    m = np.asarray(means, dt).reshape(-1, 3)
    c = np.asarray(covs, dt).reshape(-1, 6)
    o = np.asarray(opacities, dt).reshape(-1)
    R, B = int(resolution), int(num_blocks)
    f = np.float32
    # compute_voxel_field.cu:31-47, in float32 as the kernel computes them
    idx = np.arange(R)
    coord = (f(-1.0) + (f(2.0) * idx.astype(f)) / f(R - 1)).astype(f)
    bs = f(2.0) / f(B)
    blk = ((coord + f(1.0)) / bs).astype(np.int64)
    relax = f(relax_ratio)
    lo = (f(-1.0) + blk.astype(f) * bs) - bs * relax
    hi = (f(-1.0) + (blk + 1).astype(f) * bs) + bs * relax
    # compute_voxel_field.cu:6-23: the inverse covariance by cofactors
    a, b, cc, d, e, ff = (c[:, k] for k in range(6))
    det = a * d * ff + 2 * e * cc * b - e * e * a - cc * cc * d - b * b * ff
    inv_det = dt(1.0) / (det + dt(1e-24))
    ia, ib, ic = (d * ff - e * e) * inv_det, (e * cc - b * ff) * inv_det, (e * b - cc * d) * inv_det
    id_, ie, if_ = (a * ff - cc * cc) * inv_det, (b * cc - e * a) * inv_det, (a * d - b * b) * inv_det
    out = np.zeros((R, R, R), dt)
    inx = [(m[:, 0] >= lo[i]) & (m[:, 0] <= hi[i]) for i in range(R)]
    iny = [(m[:, 1] >= lo[j]) & (m[:, 1] <= hi[j]) for j in range(R)]
    inz = [(m[:, 2] >= lo[k]) & (m[:, 2] <= hi[k]) for k in range(R)]
    X = coord.astype(dt)
    for k in range(R):
        for j in range(R):
            for i in range(R):
                sel = np.nonzero(inx[i] & iny[j] & inz[k])[0]
                if sel.size == 0:
                    continue
                dx, dy, dz = X[i] - m[sel, 0], X[j] - m[sel, 1], X[k] - m[sel, 2]
                power = dt(-0.5) * (dx * dx * ia[sel] + dy * dy * id_[sel] + dz * dz * if_[sel]) \
                    - dx * dy * ib[sel] - dx * dz * ic[sel] - dy * dz * ie[sel]
                power = np.where(power > 0, dt(-1e10), power)
                terms = o[sel] * np.exp(power)
                acc = dt(0.0)
                for t in terms:  # Gaussian order, as the kernel sums
                    acc = dt(acc + t)
                out[k, j, i] = acc
    return out
