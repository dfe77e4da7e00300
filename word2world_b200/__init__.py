"""word2world_b200 -- sm_100a Gaussian rasterizer, drop-in for Word2World's
``cudaForwardBackwardRenderer._C``.

``word2world_b200._C`` exports ``rasterize_gaussians`` and
``rasterize_gaussians_backward`` with the reference extension's positional
signatures (reference ``ext.cpp:5-7``), implemented by the C ABI in
``include/w2w_raster.h`` (``libw2w_raster.so``).  ``renderer`` holds the
autograd wrapper and ``Renderer`` shim of the reference's ``Renderer.py``.

There is no CPU fallback: importing the package without the built CUDA
extension raises ImportError.
"""
from __future__ import annotations

import os

import torch  # noqa: F401  (the extension links libtorch)

_HERE = os.path.dirname(os.path.abspath(__file__))

try:
    from . import _C  # noqa: E402
except ImportError as e:  # pragma: no cover - exercised only without a build
    raise ImportError(
        "word2world_b200: the CUDA extension is not built (run `python word2world_b200/build.py`); "
        f"there is no CPU fallback. ({e})") from e

LIB_PATH = os.path.join(_HERE, "libw2w_raster.so")

__all__ = ["_C", "LIB_PATH"]
