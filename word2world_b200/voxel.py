"""Voxel occupancy field of a Gaussian set, the input of the reference's mesh
extraction (``computeVoxelFeildsCuda``, ``compute_voxel_field_wrapper.py:79-103``,
kernel ``compute_voxel_field.cu:25-124``).

``voxel_field(means, covs, opacities, resolution, num_blocks, relax_ratio)``
takes device tensors (means [N,3] normalised into [-1, 1]^3, covariances
[N,6] as xx, xy, xz, yy, yz, zz, opacities [N] or [N,1]) and returns the
[R, R, R] field on the device, laid out as the reference's wrapper returns it
(x fastest in memory).  The reference's wrapper copies to and from the host
around its kernel; ``computeVoxelFeildsCuda`` keeps that signature and
result device.
"""
from __future__ import annotations

import torch

from . import _C


def voxel_field(means, covs, opacities, resolution: int, num_blocks: int, relax_ratio: float):
    return _C.voxel_field(means.float().contiguous(), covs.float().contiguous(),
                          opacities.float().reshape(-1).contiguous(), int(resolution), int(num_blocks),
                          float(relax_ratio))


def computeVoxelFeildsCuda(means, covs, opacities, resolution, num_blocks, relax_ratio):  # noqa: N802
    """The reference wrapper's name and argument order; the field is returned
    on ``means``' device."""
    dev = means.device
    cuda = lambda t: t.to("cuda") if not t.is_cuda else t
    occ = voxel_field(cuda(means), cuda(covs), cuda(opacities), resolution, num_blocks, relax_ratio)
    return occ.to(dev)
