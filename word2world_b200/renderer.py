"""Autograd wrapper and renderer shim with the reference's Python interface.

``_render_gaussians_inline`` restates ``Renderer.py:28-110``: same argument
list, same return tuple ``(color, radii, depth, alpha)``, same gradient
routing (``dL/dmeans2D`` to the ``means2D`` placeholder, the densification
signal).  Differences, all opt-in through trailing keywords:

* ``image_height`` / ``image_width`` (the reference renders a fixed 800x800
  and derives its focal length from 800, ``Renderer.py:39-40``); the defaults
  keep 800;
* ``grad_mode="reference"`` (the reference backward's formulas) or
  ``"exact"`` (the derivative of the forward);
* ``compat_spill`` (the reference's key-emission rectangle; default on).

``Renderer`` restates ``Renderer.render`` (``Renderer.py:119-192``) over a
structure-of-arrays parameter store instead of one Python object per Gaussian.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch

from . import _C

GRAD_MODES = {"reference": 0, "exact": 1}


def fill_missing_attributes(means3D, shs, colors_precomp, scales, rotations, cov3D_precomp):
    """Empty tensors for absent optional inputs (``Renderer.py:8-23``)."""
    empty = lambda: torch.empty(0, device=means3D.device, dtype=torch.float32)
    return (shs if shs is not None else empty(), colors_precomp if colors_precomp is not None else empty(),
            scales if scales is not None else empty(), rotations if rotations is not None else empty(),
            cov3D_precomp if cov3D_precomp is not None else empty())


def _image_grads(g_color, g_depth, g_alpha, alpha):
    """The upstream image gradients as the binding takes them: colour always
    (zeros when only depth / alpha carry a loss), depth and alpha empty when
    no loss reaches them (read as zero by the kernels, no zero-filled planes)."""
    empty = alpha.new_empty(0)
    H, W = alpha.shape[-2], alpha.shape[-1]
    g_color = g_color.contiguous() if g_color is not None else alpha.new_zeros(3, H, W)
    return (g_color, g_depth.contiguous() if g_depth is not None else empty,
            g_alpha.contiguous() if g_alpha is not None else empty)


class _RasterizeGaussians(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means3D, means2D, sh, colors_precomp, opacities, scales, rotations, cov3Ds_precomp, bg,
                scale_modifier, viewmatrix, projmatrix, tanfovx, tanfovy, sh_degree, campos, prefiltered, debug,
                image_height, image_width, grad_mode, compat_spill):
        focal_x = image_width / (2.0 * tanfovx)
        focal_y = image_height / (2.0 * tanfovy)
        num_rend, color, depth, alpha, radii, geom, binb, img = _C.rasterize_gaussians(
            sh, focal_y, scales, means3D, projmatrix, sh_degree, opacities, rotations, campos, viewmatrix, focal_x,
            image_height, image_width, bg, compat_spill)
        ctx.num_rend = num_rend
        ctx.bg = bg
        ctx.scale_mod = scale_modifier
        ctx.vmat = viewmatrix
        ctx.pmat = projmatrix
        ctx.fx = tanfovx
        ctx.fy = tanfovy
        ctx.sh_deg = sh_degree
        ctx.campos = campos
        ctx.debug = debug
        ctx.grad_mode = grad_mode
        ctx.save_for_backward(colors_precomp, means3D, scales, rotations, cov3Ds_precomp, radii, sh, geom, binb, img,
                              alpha)
        ctx.mark_non_differentiable(radii)
        ctx.set_materialize_grads(False)  # an output without a gradient reaches the kernels as none
        return color, radii, depth, alpha

    @staticmethod
    def backward(ctx, g_color, g_radii, g_depth, g_alpha):
        (colors_precomp, means3D, scales, rotations, cov3Ds_precomp, radii, sh, geom, binb, img,
         alpha) = ctx.saved_tensors
        g_color, g_depth, g_alpha = _image_grads(g_color, g_depth, g_alpha, alpha)
        g_means2D, g_colors, g_opac, g_means3D, g_cov3D, g_sh, g_scales, g_rots = _C.rasterize_gaussians_backward(
            ctx.bg, means3D, radii, colors_precomp, scales, rotations, ctx.scale_mod, cov3Ds_precomp, ctx.vmat,
            ctx.pmat, ctx.fx, ctx.fy, g_color, g_depth, g_alpha, sh,
            ctx.sh_deg, ctx.campos, geom, ctx.num_rend, binb, img, alpha, ctx.debug, ctx.grad_mode)
        return (g_means3D, g_means2D, g_sh, None if colors_precomp.numel() == 0 else g_colors, g_opac, g_scales,
                g_rots, None if cov3Ds_precomp.numel() == 0 else g_cov3D,
                None, None, None, None, None, None, None, None, None, None, None, None, None, None)


def _render_gaussians_inline(means3D, means2D, shs, colors_precomp, opacity, scales, rotations, cov3D_precomp, bg,
                             scale_modifier, viewmatrix, projmatrix, tanfovx, tanfovy, sh_degree, campos,
                             prefiltered=False, debug=False, image_height=800, image_width=800,
                             grad_mode="reference", compat_spill=True):
    """``Renderer.py:28-110``: rasterize and return ``(color, radii, depth, alpha)``."""
    scale_modifier = 1  # the reference overrides it (Renderer.py:37)
    shs, colors_precomp, scales, rotations, cov3D_precomp = fill_missing_attributes(
        means3D, shs, colors_precomp, scales, rotations, cov3D_precomp)
    if grad_mode not in GRAD_MODES:
        raise ValueError(f"grad_mode must be one of {sorted(GRAD_MODES)}")
    return _RasterizeGaussians.apply(means3D, means2D, shs, colors_precomp, opacity, scales, rotations,
                                     cov3D_precomp, bg, scale_modifier, viewmatrix, projmatrix, tanfovx, tanfovy,
                                     sh_degree, campos, prefiltered, debug, int(image_height), int(image_width),
                                     GRAD_MODES[grad_mode], bool(compat_spill))


class _Activate(torch.autograd.Function):
    """The activation preamble of ``Renderer.render`` (``Renderer.py:164-167``:
    sigmoid opacity, exp scales, normalised quaternion, concatenated SH) as
    one fused kernel each way; the forward is bit-identical to the torch
    operations the reference runs."""

    @staticmethod
    def forward(ctx, opacity_logit, svec, quaternion, sh_dc, sh_ac):
        opacity, scales, rotations, shs = _C.activate(opacity_logit, svec, quaternion, sh_dc, sh_ac)
        ctx.save_for_backward(opacity, scales, quaternion)
        ctx.rows = shs.shape[1]
        return opacity, scales, rotations, shs

    @staticmethod
    def backward(ctx, g_opacity, g_scales, g_rotations, g_shs):
        opacity, scales, quaternion = ctx.saved_tensors
        z = lambda g, like: torch.zeros_like(like) if g is None else g
        P = opacity.shape[0]
        d_logit, d_svec, d_quat, d_dc, d_ac = _C.activate_backward(
            z(g_opacity, opacity), z(g_scales, scales), z(g_rotations, quaternion),
            z(g_shs, torch.empty(P, ctx.rows, 3, device=opacity.device)), opacity, scales, quaternion)
        return d_logit, d_svec, d_quat, d_dc, d_ac


def activate(opacity_logit, svec, quaternion, sh_dc, sh_ac):
    """(opacity, scales, rotations, shs) from the raw parameters, differentiable."""
    return _Activate.apply(opacity_logit, svec, quaternion, sh_dc, sh_ac)


class _RasterizeRaw(torch.autograd.Function):
    """``Renderer.render``'s preamble and rasterization in one forward and one
    backward call on the raw parameters (opacity logits, log-scales,
    unnormalised quaternions, split SH): the projection pass activates them
    as it reads them, with the same arithmetic as ``activate`` (the image is
    bit-identical to ``activate`` followed by ``_render_gaussians_inline``),
    and the per-Gaussian backward applies the activations' chain rule before
    it stores.  Reference-formula gradients only."""

    @staticmethod
    def forward(ctx, means3D, means2D, sh_dc, sh_ac, opacity_logit, svec, quaternion, bg, viewmatrix, projmatrix,
                tanfovx, tanfovy, sh_degree, campos, image_height, image_width, compat_spill, densification=None):
        focal_x = image_width / (2.0 * tanfovx)
        num_rend, color, depth, alpha, radii, geom, binb, img = _C.rasterize_gaussians_raw(
            means3D, sh_dc, sh_ac, opacity_logit, svec, quaternion, viewmatrix, projmatrix, campos, focal_x,
            sh_degree, image_height, image_width, bg, compat_spill)
        ctx.num_rend = num_rend
        ctx.bg, ctx.vmat, ctx.pmat, ctx.campos = bg, viewmatrix, projmatrix, campos
        ctx.fx, ctx.fy, ctx.sh_deg = tanfovx, tanfovy, sh_degree
        ctx.dens = densification  # a DensificationStats the backward updates, or None
        ctx.save_for_backward(means3D, sh_dc, sh_ac, opacity_logit, svec, quaternion, radii, geom, binb, img, alpha)
        ctx.mark_non_differentiable(radii)
        ctx.set_materialize_grads(False)
        return color, radii, depth, alpha

    @staticmethod
    def backward(ctx, g_color, g_radii, g_depth, g_alpha):
        means3D, sh_dc, sh_ac, opacity_logit, svec, quaternion, radii, geom, binb, img, alpha = ctx.saved_tensors
        g_color, g_depth, g_alpha = _image_grads(g_color, g_depth, g_alpha, alpha)
        g_means2D, g_means3D, g_dc, g_ac, g_logit, g_svec, g_quat = _C.rasterize_gaussians_backward_raw(
            ctx.bg, means3D, sh_dc, sh_ac, opacity_logit, svec, quaternion, radii, ctx.vmat, ctx.pmat, ctx.campos,
            ctx.fx, ctx.fy, ctx.sh_deg, g_color, g_depth, g_alpha, geom,
            ctx.num_rend, binb, img, alpha,
            dens_accum=ctx.dens.mean_gradient_accum if ctx.dens is not None else None,
            dens_counter=ctx.dens.counter if ctx.dens is not None else None)
        return (g_means3D, g_means2D, g_dc, g_ac, g_logit, g_svec, g_quat,
                None, None, None, None, None, None, None, None, None, None, None)


@dataclass
class GaussianParams:
    """Raw per-Gaussian parameters as structure-of-arrays tensors (the
    reference keeps one ``GaussianPrimitive`` object per Gaussian,
    ``primitives.py:54-86``)."""
    mean: torch.Tensor        # [P,3]
    sh_dc: torch.Tensor       # [P,1,3]
    sh_ac: torch.Tensor       # [P,15,3]
    opacity: torch.Tensor     # [P,1] logits
    svec: torch.Tensor        # [P,3] log-scales
    quaternion: torch.Tensor  # [P,4] (w, x, y, z)

    @staticmethod
    def from_scene(scene, device="cuda", requires_grad=True):
        t = lambda a: torch.tensor(a, device=device, dtype=torch.float32).requires_grad_(requires_grad)
        return GaussianParams(t(scene.mean), t(scene.sh_dc), t(scene.sh_ac), t(scene.opacity), t(scene.svec),
                              t(scene.quaternion))

    def parameters(self):
        return [self.mean, self.sh_dc, self.sh_ac, self.opacity, self.svec, self.quaternion]

    def save_ply(self, path):
        """The reference's PLY layout (``GaussianIO.save_as_ply``)."""
        from .ply import save_ply
        save_ply(path, self.mean, self.sh_dc, self.sh_ac, self.opacity, self.svec, self.quaternion)

    @staticmethod
    def load_ply(path, device="cuda", requires_grad=True):
        from .ply import load_ply
        d = load_ply(path)
        t = lambda a: torch.tensor(a, device=device, dtype=torch.float32).requires_grad_(requires_grad)
        return GaussianParams(t(d["mean"]), t(d["sh_dc"]), t(d["sh_ac"]), t(d["opacity"]), t(d["svec"]),
                              t(d["quaternion"]))


class DensificationStats:
    """The training loop's densification statistics
    (``gaussians_handler.collect_densification_info``,
    ``gaussians_handler.py:116-118``): per Gaussian, the number of renders in
    which it was visible and the sum of its screen-space gradient norms.
    ``collect`` updates both in one fused pass, with no host synchronisation
    (the reference indexes with a boolean mask)."""

    def __init__(self, P: int, device="cuda"):
        self.mean_gradient_accum = torch.zeros((P, 1), dtype=torch.float32, device=device)
        self.counter = torch.zeros((P, 1), dtype=torch.float32, device=device)

    def collect(self, viewspace_point_tensor, radii):
        """``viewspace_point_tensor``: the render's ``accum_grads`` (its
        ``.grad`` is read) or that gradient itself; ``radii``: the render's
        radii (visible = radius > 0, the reference's ``avaialble_pts``)."""
        g = viewspace_point_tensor.grad if viewspace_point_tensor.grad is not None else viewspace_point_tensor
        _C.densification_stats(g.detach(), radii.to(torch.int32), self.mean_gradient_accum, self.counter)


class Renderer:
    """``Renderer.render`` (``Renderer.py:119-192``) over ``GaussianParams``.

    ``sh_degree`` defaults to 0 as in the reference call (``Renderer.py:170``).
    Unlike the reference, ``image_width`` / ``image_height`` are honoured.
    """

    def __init__(self, params: GaussianParams, sh_degree: int = 0, grad_mode: str = "reference",
                 compat_spill: bool = True, densification: "DensificationStats | None" = None):
        """``densification``: statistics every render's backward accumulates
        (reference-formula gradients), in the per-Gaussian pass itself,
        instead of a ``collect`` call after each backward (the reference's
        trainer collects after the backward, ``GaussianTrainer.py:119``)."""
        if densification is not None and grad_mode != "reference":
            raise ValueError("fused densification statistics come with reference-formula gradients; with "
                             "grad_mode='exact' call DensificationStats.collect after the backward")
        self.params = params
        self.densification = densification
        self.sh_degree = sh_degree
        self.grad_mode = grad_mode
        self.compat_spill = compat_spill
        self._bg = None  # the white background (Renderer.py:169), kept across calls
        self._zeros = None  # the screen-space points' zeros, kept across calls

    def render(self, FoVx, FoVy, world_view_transform, full_proj_transform, camera_center, image_width,
               image_height):
        p = self.params
        # the screen-space points (Renderer.py:121-126): zeros whose gradient
        # the backward fills.  Each call gets a fresh leaf (its own .grad) over
        # one zero buffer kept across calls, which nothing writes (torch
        # refuses in-place writes to a leaf that requires grad), instead of a
        # new zero-filled tensor per call
        z = self._zeros
        if z is None or z.shape != p.mean.shape or z.device != p.mean.device or z.dtype != p.mean.dtype:
            z = self._zeros = torch.zeros_like(p.mean)
        accum_grads = z.detach().requires_grad_(True)
        accum_grads.retain_grad()
        tanfovx = math.tan(float(FoVx) * 0.5)
        tanfovy = math.tan(float(FoVy) * 0.5)
        if self._bg is None or self._bg.device != p.mean.device:
            self._bg = torch.ones(3, dtype=torch.float32, device=p.mean.device)
        bg = self._bg
        if self.grad_mode == "reference":
            # activation preamble (Renderer.py:164-167) folded into the projection
            # pass and the per-Gaussian backward
            image, radii, _, _ = _RasterizeRaw.apply(
                p.mean, accum_grads, p.sh_dc, p.sh_ac, p.opacity, p.svec, p.quaternion, bg, world_view_transform,
                full_proj_transform, tanfovx, tanfovy, self.sh_degree, camera_center, int(image_height),
                int(image_width), bool(self.compat_spill), self.densification)
            available = radii > 0
            return {"image": image, "accum_grads": accum_grads, "avaialble_pts": available,
                    "available_pts": available}
        # activation preamble (Renderer.py:164-167), one fused kernel each way
        activated_opacity, activated_scales, rotations, shs = activate(p.opacity, p.svec, p.quaternion, p.sh_dc,
                                                                       p.sh_ac)
        image, radii, _, _ = _render_gaussians_inline(
            p.mean, accum_grads, shs, None, activated_opacity, activated_scales, rotations, None, bg, 1,
            world_view_transform, full_proj_transform, tanfovx, tanfovy, self.sh_degree, camera_center, False,
            False, image_height=int(image_height), image_width=int(image_width), grad_mode=self.grad_mode,
            compat_spill=self.compat_spill)
        available = radii > 0
        # the reference's result keys, including its spelling of "avaialble_pts"
        return {"image": image, "accum_grads": accum_grads, "avaialble_pts": available, "available_pts": available}
