"""Build recipe for ``oracle/_ref``: the unmodified reference rasterizer extension.

Test infrastructure only.  Compiles the reference's own CUDA/C++ sources
(``cudaForwardBackwardRenderer/{gaussianRasterizer,gaussianForwardPass,backward,
rasterize_points,projection,ADRculling,pixelGaussiansFull,gaussianTiles,prepareSort,
gradientPass}.cu`` and ``ext.cpp``, the list in ``cudaForwardBackwardRenderer/setup.py:11-23``)
in place, with the vendored GLM headers on the include path
(``setup.py:25``), for sm_100a.  Nothing is copied: the sources are read where
they lie and every output goes to ``oracle/_ref/``.  The reference's own
``setup.py`` is not run; this script drives ``torch.utils.cpp_extension`` with
the same sources and include path.

The result ``oracle/_ref/w2w_reference_C.so`` exposes the reference's two entry
points ``rasterize_gaussians`` / ``rasterize_gaussians_backward``
(``cudaForwardBackwardRenderer/ext.cpp:5-7``).  It is loaded only by the GPU
parity tests, the golden-fixture generator and ``bench.py --impl reference``.

Usage: python oracle/build_ref.py [--ref-root PATH]; the default location of
the reference checkout is $W2W_REFERENCE_ROOT, else /root/reference.
"""
import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
REFERENCE_ROOT = os.environ.get("W2W_REFERENCE_ROOT", "/root/reference")
MODULE_NAME = "w2w_reference_C"
SOURCES = [
    "gaussianRasterizer.cu", "gaussianForwardPass.cu", "backward.cu",
    "rasterize_points.cu", "projection.cu", "ADRculling.cu",
    "pixelGaussiansFull.cu", "gaussianTiles.cu", "prepareSort.cu",
    "gradientPass.cu", "ext.cpp",
]


def build(ref_root=REFERENCE_ROOT, verbose=False):
    src_dir = os.path.join(ref_root, "cudaForwardBackwardRenderer")
    if not os.path.isdir(src_dir):
        raise FileNotFoundError(f"reference sources not found at {src_dir}")
    os.makedirs(OUT, exist_ok=True)
    os.environ["TORCH_CUDA_ARCH_LIST"] = "10.0a"
    os.environ.setdefault("MAX_JOBS", str(os.cpu_count() or 4))
    from torch.utils.cpp_extension import load
    mod = load(
        name=MODULE_NAME,
        sources=[os.path.join(src_dir, s) for s in SOURCES],
        extra_include_paths=[os.path.join(src_dir, "GLMLibrary")],
        build_directory=OUT,
        verbose=verbose,
    )
    return mod


def so_path():
    return os.path.join(OUT, MODULE_NAME + ".so")


VOXEL_SO = os.path.join(OUT, "compute_voxel_field.so")


def build_voxel(ref_root=REFERENCE_ROOT):
    """The reference's voxel-field kernel (``compute_voxel_field.cu``) as a
    shared library exporting ``compute_voxel_field_cuda``, compiled from its
    one source file where it lies.  The source marks the export with the
    Windows-only ``__declspec(dllexport)``; the command line defines that away."""
    import subprocess
    src = os.path.join(ref_root, "compute_voxel_field.cu")
    if not os.path.exists(src):
        raise FileNotFoundError(src)
    os.makedirs(OUT, exist_ok=True)
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    subprocess.run([nvcc, "-O3", "-shared", "-Xcompiler", "-fPIC", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-D__declspec(x)=", src, "-o", VOXEL_SO], check=True)
    return VOXEL_SO


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=REFERENCE_ROOT)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    build(a.ref_root, a.v)
    build_voxel(a.ref_root)
    print(so_path(), os.path.exists(so_path()), VOXEL_SO, os.path.exists(VOXEL_SO))
    sys.exit(0)
