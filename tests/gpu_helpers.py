"""GPU-side helpers for the parity tests: run the CUDA rasterizer through its
torch binding and unpack its state buffers into numpy arrays named like the
oracle's outputs."""
from __future__ import annotations

import numpy as np
import torch

from word2world_b200 import _C


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def _field(buf_np, off, dtype, count):
    nbytes = count * np.dtype(dtype).itemsize
    return buf_np[off:off + nbytes].view(dtype).copy()


def unpack_geometry(geom, P):
    g = geom.cpu().numpy()
    o = lambda n: _C.geometry_offset(P, n)
    out = dict(
        depth=_field(g, o("depth"), np.float32, P),
        clamped=_field(g, o("clamped"), np.uint8, 3 * P).reshape(P, 3),
        means2D=_field(g, o("means2D"), np.float32, 2 * P).reshape(P, 2),
        cov3D=_field(g, o("cov3D"), np.float32, 6 * P).reshape(P, 6),
        conic_opac=_field(g, o("conic_opacity"), np.float32, 4 * P).reshape(P, 4),
        rgb=_field(g, o("rgb"), np.float32, 3 * P).reshape(P, 3),
        tiles=_field(g, o("tiles_touched"), np.uint32, P),
        offsets=_field(g, o("offsets"), np.uint32, P),
        record=_field(g, o("record"), np.float32, 16 * P).reshape(P, 16),
    )
    out["header"] = _field(g, o("header"), np.uint32, 8)
    return out


def unpack_image(img, W, H):
    b = img.cpu().numpy()
    T = ((W + 15) // 16) * ((H + 15) // 16)
    o = lambda n: _C.image_offset(W, H, n)
    return dict(n_contrib=_field(b, o("n_contrib"), np.uint32, W * H).reshape(H, W),
                ranges=_field(b, o("ranges"), np.uint32, 2 * T).reshape(T, 2),
                T_final=_field(b, o("T_final"), np.float32, W * H).reshape(H, W),
                tile_max=_field(b, o("tile_max"), np.uint32, T))


def forward(arrays, cam, degree=3, compat_spill=True, bg=(1.0, 1.0, 1.0), focal_x=None, W=None, H=None):
    means3D, opac, scales, rots, shs = arrays
    W = cam.width if W is None else W
    H = cam.height if H is None else H
    fx = cam.focal_x if focal_x is None else focal_x
    out = _C.rasterize_gaussians(dev(shs), float(cam.focal_y), dev(scales), dev(means3D), dev(cam.projmatrix),
                                 int(degree), dev(opac), dev(rots), dev(cam.campos), dev(cam.viewmatrix), float(fx),
                                 int(H), int(W), dev(np.asarray(bg, np.float32)), bool(compat_spill))
    R, color, depth, alpha, radii, geom, binb, img = out
    P = means3D.shape[0]
    res = unpack_geometry(geom, P)
    res.update(unpack_image(img, W, H))
    keys = _C.binning_keys64(binb, R, H, W).cpu().numpy().view(np.uint64) if R > 0 else np.zeros(0, np.uint64)
    b = binb.cpu().numpy()
    # the point list: the state is laid out for R, or for a planned render's capacity
    LR = _C.binning_layout_count(R, binb, H, W)
    pl = _field(b, _C.binning_offset(LR, W, H, "vals_a"), np.uint32, R) if R > 0 else np.zeros(0, np.uint32)
    res.update(num_rendered=int(R), color=color.cpu().numpy(), depth_img=depth.cpu().numpy(),
               alpha=alpha.cpu().numpy(), radii=radii.cpu().numpy(), keys=keys, point_list=pl,
               layout_count=int(LR), _tensors=dict(geom=geom, binb=binb, img=img, alpha=alpha, radii=radii))
    return res


def backward(fwd, arrays, cam, dL_dcolor, dL_ddepth=None, dL_dalpha=None, degree=3, grad_mode=0, bg=(1.0, 1.0, 1.0),
             tan=None):
    means3D, opac, scales, rots, shs = arrays
    t = fwd["_tensors"]
    H, W = dL_dcolor.shape[1:]
    dLd = np.zeros((1, H, W), np.float32) if dL_ddepth is None else dL_ddepth
    dLa = np.zeros((1, H, W), np.float32) if dL_dalpha is None else dL_dalpha
    tfx, tfy = (cam.tanfovx, cam.tanfovy) if tan is None else tan
    empty = torch.empty(0, device="cuda")
    g = _C.rasterize_gaussians_backward(
        dev(np.asarray(bg, np.float32)), dev(means3D), t["radii"], empty, dev(scales), dev(rots), 1.0, empty,
        dev(cam.viewmatrix), dev(cam.projmatrix), float(tfx), float(tfy), dev(dL_dcolor), dev(dLd), dev(dLa),
        dev(shs), int(degree), dev(cam.campos), t["geom"], fwd["num_rendered"], t["binb"], t["img"], t["alpha"],
        False, int(grad_mode))
    names = ["dL_dmeans2D", "dL_dcolors", "dL_dopacity", "dL_dmeans3D", "dL_dcov3D", "dL_dsh", "dL_dscales",
             "dL_drotations"]
    return {k: v.cpu().numpy() for k, v in zip(names, g)}


class tuned:
    """Tuning knobs set for the duration (word2world_b200.autotune)."""

    def __init__(self, **knobs):
        self.knobs = knobs

    def __enter__(self):
        from word2world_b200 import autotune
        self.prev = autotune.apply(self.knobs)
        return self

    def __exit__(self, *exc):
        from word2world_b200 import autotune
        autotune.apply(self.prev)
