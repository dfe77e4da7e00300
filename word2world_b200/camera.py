"""Camera conventions of the reference trainer, restated.

The reference builds one orbit camera per training view
(``GaussianTrainer.py:50-83``) and hands the rasterizer

* ``viewmatrix`` = transpose of ``inv(c2w)`` with rotation rows 1 and 2 and the
  translation negated (``GaussianTrainer.py:76-79``);
* ``projmatrix`` = ``viewmatrix @ P^T`` with ``P`` from
  ``misc_utils.get_projection_matrix`` (``misc_utils.py:143-173``, z_sign=+1);
* ``campos`` = **minus** the camera position (``GaussianTrainer.py:83``);
* ``tanfovx = tan(FoVx/2)``, ``tanfovy = tan(FoVy/2)`` (``Renderer.py:133-134``)
  with ``FoVx`` from ``utils_for_camera.compute_fovx`` (``utils_for_camera.py:11-12``);
* near 0.01, far 100, fovy 49.1 degrees (``DynamicCamera.py:5``).

Matrices are float32 row-major 4x4 arrays whose memory the kernels read
column-major, exactly as the reference extension does.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class Camera:
    viewmatrix: np.ndarray   # [4,4] float32, as passed to rasterize_gaussians
    projmatrix: np.ndarray   # [4,4] float32
    campos: np.ndarray       # [3] float32 (minus the camera position)
    fovx: float
    fovy: float
    width: int
    height: int

    @property
    def tanfovx(self) -> float:
        return math.tan(self.fovx * 0.5)

    @property
    def tanfovy(self) -> float:
        return math.tan(self.fovy * 0.5)

    @property
    def focal_x(self) -> float:
        """Horizontal focal length in pixels, W / (2 tan(fovx/2))."""
        return self.width / (2.0 * self.tanfovx)

    @property
    def focal_y(self) -> float:
        return self.height / (2.0 * self.tanfovy)


def _normalize(v: np.ndarray) -> np.ndarray:
    v = np.asarray(v, dtype=np.float32)
    n = np.sqrt(np.maximum(np.dot(v, v), np.float32(1e-20)))
    return (v / n).astype(np.float32)


def projection_matrix(z_near: float, z_far: float, fov_x: float, fov_y: float) -> np.ndarray:
    """``misc_utils.get_projection_matrix`` (misc_utils.py:143-173)."""
    p = np.zeros((4, 4), dtype=np.float32)
    p[0, 0] = 1.0 / math.tan(fov_x / 2.0)
    p[1, 1] = 1.0 / math.tan(fov_y / 2.0)
    p[2, 2] = z_far / (z_far - z_near)
    p[2, 3] = -(z_far * z_near) / (z_far - z_near)
    p[3, 2] = 1.0
    return p


def compute_fovx(fovy: float, width: int, height: int) -> float:
    """``utils_for_camera.compute_fovx`` in float32 (utils_for_camera.py:11-12)."""
    fy = np.float32(fovy)
    return float(np.float32(2.0) * np.arctan(np.tan(fy / np.float32(2.0)) * np.float32(width) / np.float32(height)))


def orbit_camera(azimuth_deg: float, elevation_deg: float, radius: float, width: int, height: int,
                 fovy_deg: float = 49.1, near: float = 0.01, far: float = 100.0) -> Camera:
    """One orbit view as ``GaussianTrainer.render_training_views`` builds it
    (GaussianTrainer.py:50-83), target at the origin."""
    el = math.radians(elevation_deg)
    az = math.radians(azimuth_deg)
    x = radius * math.cos(el) * math.sin(az)
    y = -radius * math.sin(el)
    z = radius * math.cos(el) * math.cos(az)
    campos = np.array([x, y, z], dtype=np.float64)
    forward = _normalize(campos.astype(np.float32))
    up = np.array([0, 1, 0], dtype=np.float32)
    right = _normalize(np.cross(up, forward))
    up = _normalize(np.cross(forward, right))
    pose = np.eye(4, dtype=np.float32)
    pose[:3, :3] = np.stack([right, up, forward], axis=1)
    pose[:3, 3] = campos.astype(np.float32)
    fovy = float(np.float32(math.radians(fovy_deg)))
    fovx = compute_fovx(fovy, width, height)
    w2c = np.linalg.inv(pose.astype(np.float64)).astype(np.float32)
    w2c[1:3, :3] *= -1
    w2c[:3, 3] *= -1
    view = np.ascontiguousarray(w2c.T)
    proj_t = np.ascontiguousarray(projection_matrix(near, far, fovx, fovy).T)
    full = (view.astype(np.float32) @ proj_t.astype(np.float32)).astype(np.float32)
    cc = (-pose[:3, 3]).astype(np.float32)
    return Camera(viewmatrix=view, projmatrix=np.ascontiguousarray(full), campos=cc,
                  fovx=fovx, fovy=fovy, width=width, height=height)


def orbit_views(n_views: int, radius: float, width: int, height: int, elevation_deg: float = 0.0,
                azimuth0_deg: float = 0.0) -> list:
    """``n_views`` azimuths spaced 360/n_views apart (0/90/180/270 for 4)."""
    step = 360.0 / n_views
    return [orbit_camera(azimuth0_deg + k * step, elevation_deg, radius, width, height)
            for k in range(n_views)]


def crop_embed(cam: Camera, frame: int = 800) -> Camera:
    """Re-express a W'xW' camera so that, rendered into a ``frame`` x ``frame``
    image, its pixels land in the top-left W'xW' crop.

    Clip coordinates are remapped x' = s x + (s-1) w, y' = s y + (s-1) w with
    s = W'/frame; z and w are untouched, so depth keys are unchanged.  The
    focal length stays the W' one, so the EWA Jacobian is the W' one.  Used to
    drive a rasterizer whose resolution is fixed at ``frame``.
    """
    assert cam.width == cam.height and cam.width <= frame
    s = cam.width / frame
    A = np.eye(4, dtype=np.float64)
    A[0, 0] = s
    A[0, 3] = s - 1.0
    A[1, 1] = s
    A[1, 3] = s - 1.0
    full = (cam.projmatrix.astype(np.float64) @ A.T).astype(np.float32)
    return Camera(viewmatrix=cam.viewmatrix.copy(), projmatrix=np.ascontiguousarray(full),
                  campos=cam.campos.copy(), fovx=cam.fovx, fovy=cam.fovy, width=frame, height=frame)
