"""In-tree build of the rasterizer for sm_100a.

* ``libw2w_raster.so`` -- the CUDA kernels and the C ABI of
  ``include/w2w_raster.h`` (nvcc, ``-gencode arch=compute_100a,code=sm_100a``,
  static CUDA runtime, no torch dependency);
* ``_C<ext suffix>`` -- the pybind torch binding (g++ against torch's headers),
  linked to ``libw2w_raster.so`` through ``$ORIGIN``.

Both land next to this file so they travel with the source tree.  Rebuilds only
what is older than its sources.  ``python word2world_b200/build.py [--force]`` (run as a
script: importing the package needs the extension this builds).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libw2w_raster.so")
CUDA_SOURCES = ["preprocess.cu", "duplicate.cu", "sort.cu", "binning.cu", "blend.cu", "backward.cu", "scan.cu", "activate.cu",
                "densify.cu", "voxel.cu", "groupsum.cu", "capi.cu", "timing.cu"]
HEADERS = ["common.cuh", "kernels.h", "pinned_fp.h", "tile_walk.cuh", "tma.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def ext_path() -> str:
    return os.path.join(HERE, "_C" + sysconfig.get_config_var("EXT_SUFFIX"))


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build_lib(force: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "w2w_raster.h")]
    objs, todo = [], []
    for src in CUDA_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or not _newer(o, [s] + hdrs):
            todo.append([NVCC] + ARCH + NVCC_FLAGS + ["-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        list(ex.map(_run, todo))
    if force or todo or not _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs)
    return LIB


def build_ext(force: bool = False) -> str:
    import torch
    from torch.utils.cpp_extension import include_paths, library_paths

    out = ext_path()
    src = os.path.join(CSRC, "binding.cpp")
    deps = [src, LIB, os.path.join(ROOT, "include", "w2w_raster.h")]
    if not force and _newer(out, deps):
        return out
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    inc = include_paths() + [sysconfig.get_paths()["include"], "/usr/local/cuda/include"]
    libdirs = library_paths()
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           "-DTORCH_EXTENSION_NAME=_C", "-DTORCH_API_INCLUDE_EXTENSION_H", src, "-o", out]
    cmd += [f"-I{p}" for p in inc]
    cmd += [f"-L{p}" for p in libdirs] + [f"-L{HERE}"]
    cmd += ["-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python", "-lw2w_raster"]
    cmd += ["-Wl,-rpath,$ORIGIN"] + [f"-Wl,-rpath,{p}" for p in libdirs]
    _run(cmd)
    return out


def build(force: bool = False) -> None:
    build_lib(force)
    build_ext(force)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build(a.force)
    print(LIB)
    print(ext_path())
    sys.exit(0)
