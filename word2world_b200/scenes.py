"""Seeded synthetic scenes with the benchmark's parameter distributions.

There is no dataset for this path; every workload is synthetic:

* means: unit-sphere directions x 0.5 plus N(0, 0.05^2) jitter (16,384-Gaussian
  scene), or uniform in a radius-0.6 ball (500,000-Gaussian scene);
* log-scales U[-5, -3] per axis; rotations uniform unit quaternions
  (normalised N(0, I4)); opacity logits U[-2, 2];
* SH degree 3 (16 x 3 coefficients): DC ~ N(0.5, 0.2^2), higher bands
  ~ N(0, 0.05^2);
* 4 orbit cameras at azimuth 0/90/180/270, elevation 0, radius 2.5,
  fovy 49.1 degrees, white background; upstream dL/dimage ~ N(0, 1).

``Scene`` holds the raw (pre-activation) parameters the reference keeps per
Gaussian (``primitives.py:54-86``) as structure-of-arrays float32 arrays;
``activate`` applies ``Renderer.py:164-167``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Scene:
    mean: np.ndarray        # [P,3]
    svec: np.ndarray        # [P,3] log-scales
    quaternion: np.ndarray  # [P,4] (w, x, y, z), unnormalised allowed
    opacity: np.ndarray     # [P,1] logits
    sh_dc: np.ndarray       # [P,1,3]
    sh_ac: np.ndarray       # [P,15,3]

    @property
    def P(self) -> int:
        return self.mean.shape[0]

    def activate(self):
        """(means3D, opacities, scales, rotations, shs) as Renderer.py:164-167."""
        opac = (1.0 / (1.0 + np.exp(-self.opacity.astype(np.float64)))).astype(np.float32)
        scales = np.exp(self.svec.astype(np.float64)).astype(np.float32)
        q = self.quaternion.astype(np.float64)
        q = q / np.maximum(np.linalg.norm(q, axis=1, keepdims=True), 1e-12)
        shs = np.concatenate([self.sh_dc, self.sh_ac], axis=1).astype(np.float32)
        return (np.ascontiguousarray(self.mean, dtype=np.float32), np.ascontiguousarray(opac),
                np.ascontiguousarray(scales), np.ascontiguousarray(q.astype(np.float32)),
                np.ascontiguousarray(shs))


def _sphere_dirs(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def make_scene(P: int, seed: int = 0, layout: str = "shell", radius: float | None = None,
               log_scale=(-5.0, -3.0), sh_rest: int = 15) -> Scene:
    """``layout="shell"``: directions x 0.5 + N(0, 0.05^2) jitter;
    ``layout="ball"``: uniform in a ball of ``radius`` (default 0.6)."""
    rng = np.random.default_rng(seed)
    if layout == "shell":
        r = 0.5 if radius is None else radius
        mean = _sphere_dirs(rng, P) * r + rng.normal(0.0, 0.05, size=(P, 3))
    elif layout == "ball":
        r = 0.6 if radius is None else radius
        mean = _sphere_dirs(rng, P) * (r * np.cbrt(rng.uniform(size=(P, 1))))
    else:
        raise ValueError(layout)
    svec = rng.uniform(log_scale[0], log_scale[1], size=(P, 3))
    quat = rng.normal(size=(P, 4))
    quat = quat / np.linalg.norm(quat, axis=1, keepdims=True)
    opac = rng.uniform(-2.0, 2.0, size=(P, 1))
    sh_dc = rng.normal(0.5, 0.2, size=(P, 1, 3))
    sh_ac = rng.normal(0.0, 0.05, size=(P, sh_rest, 3))
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    return Scene(f(mean), f(svec), f(quat), f(opac), f(sh_dc), f(sh_ac))


def upstream_grads(n_views: int, H: int, W: int, seed: int = 1):
    """dL/dimage ~ N(0,1) [3,H,W] per view; dL/ddepth = dL/dalpha = 0."""
    rng = np.random.default_rng(seed)
    return [np.ascontiguousarray(rng.normal(size=(3, H, W)), dtype=np.float32) for _ in range(n_views)]


# Named workloads -----------------------------------------------------------

def scene_16k(seed: int = 0) -> Scene:
    """16,384 Gaussians on a 0.5 shell (rendered at 256x256, 4 views)."""
    return make_scene(16384, seed=seed, layout="shell")


def scene_500k(seed: int = 0) -> Scene:
    """500,000 Gaussians in a 0.6 ball (rendered at 512x512, 4 views)."""
    return make_scene(500000, seed=seed, layout="ball")


# Isolated sort / scan stage workload ------------------------------------------

def sort_workload(n: int, seed: int = 0, num_tiles: int = 4096, zipf_a: float = 1.2):
    """(keys u64[n], values u32[n]): key = tile << 32 | float32 depth bits with
    tile ids in [0, num_tiles) drawn from a Zipf(zipf_a) skew (p ~ 1/(k+1)^a),
    depths U[0.5, 4.5]; value = position (the 1024x1024, 16x16-tile case)."""
    rng = np.random.default_rng(seed)
    p = 1.0 / np.power(np.arange(1, num_tiles + 1, dtype=np.float64), zipf_a)
    p /= p.sum()
    tiles = rng.choice(num_tiles, size=n, p=p).astype(np.uint64)
    depth = rng.uniform(0.5, 4.5, size=n).astype(np.float32)
    keys = (tiles << np.uint64(32)) | depth.view(np.uint32).astype(np.uint64)
    return keys, np.arange(n, dtype=np.uint32)


def scan_workload(n: int, seed: int = 0, lam: float = 8.0):
    """Per-Gaussian tile-touch counts ~ Poisson(lam), uint32."""
    rng = np.random.default_rng(seed)
    return rng.poisson(lam, size=n).astype(np.uint32)
