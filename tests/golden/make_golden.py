"""Generate golden vectors from the reference extension (run on a B200).

Runs the unmodified reference rasterizer (``oracle/_ref/w2w_reference_C.so``,
built by ``oracle/build_ref.py`` from the reference sources) on seeded
synthetic inputs and writes every buffer it produces:

* geometry state carved exactly as ``gaussianRasterizer.cu:145-186``
  (depth, clamped, means2D, cov3D, conic/opacity, rgb, tiles, offsets);
* binning state as ``prepareSort.cu:389-421`` (sorted ids, unsorted ids,
  unsorted keys, sorted keys);
* image state as ``gaussianRasterizer.cu:189-206`` (n_contrib, tile ranges);
* the images, radii and the eight backward outputs.

The reference renders a fixed 800x800 frame (``rasterize_points.cu:111-113``).
Cases at other resolutions are crop-embedded (``word2world_b200.camera.crop_embed``).

Usage (on a GPU box):
    python tests/golden/make_golden.py --out DIR [--full] [--cases a,b,...]
``--full`` keeps the whole 800x800 images; otherwise images are cropped to the
case's region and the case list is the small committed set.
"""
from __future__ import annotations

import argparse
import importlib.machinery
import importlib.util
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from word2world_b200 import camera, scenes  # noqa: E402

FRAME = 800


def load_reference():
    import torch  # noqa: F401  (the extension needs libtorch loaded)
    path = os.path.join(ROOT, "oracle", "_ref", "w2w_reference_C.so")
    loader = importlib.machinery.ExtensionFileLoader("w2w_reference_C", path)
    spec = importlib.util.spec_from_loader("w2w_reference_C", loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def _align128(x):
    return (x + 127) & ~127


def carve_geom(buf: np.ndarray, P: int) -> dict:
    """Fields of the reference geometry buffer (gaussianRasterizer.cu:145-186)."""
    fields = [("depth", np.float32, P), ("clamped", np.uint8, 3 * P), ("internal_radii", np.int32, P),
              ("means2D", np.float32, 2 * P), ("cov3D", np.float32, 6 * P), ("conic_opac", np.float32, 4 * P),
              ("rgb", np.float32, 3 * P), ("tiles", np.uint32, P), ("scan_tmp", np.uint8, 0),
              ("offsets", np.uint32, P)]
    out, off = {}, 0
    for name, dt, n in fields:
        a = _align128(off)
        nbytes = n * np.dtype(dt).itemsize
        out[name] = buf[a:a + nbytes].view(dt).copy()
        off = a + nbytes
    out["means2D"] = out["means2D"].reshape(P, 2)
    out["cov3D"] = out["cov3D"].reshape(P, 6)
    out["conic_opac"] = out["conic_opac"].reshape(P, 4)
    out["rgb"] = out["rgb"].reshape(P, 3)
    out["clamped"] = out["clamped"].reshape(P, 3)
    del out["scan_tmp"], out["internal_radii"]
    return out


def carve_bin(buf: np.ndarray, R: int) -> dict:
    """Binning buffer (prepareSort.cu:389-421)."""
    fields = [("point_list", np.uint32), ("unsorted_vals", np.uint32), ("unsorted_keys", np.uint64),
              ("keys", np.uint64)]
    out, off = {}, 0
    for name, dt in fields:
        a = _align128(off)
        nbytes = R * np.dtype(dt).itemsize
        out[name] = buf[a:a + nbytes].view(dt).copy()
        off = a + nbytes
    return out


def carve_img(buf: np.ndarray) -> dict:
    """Image buffer (gaussianRasterizer.cu:189-206): n_contrib[640000], ranges[2500]."""
    n = buf[0:640000 * 4].view(np.uint32).copy().reshape(FRAME, FRAME)
    a = _align128(640000 * 4)
    ranges = buf[a:a + 2500 * 8].view(np.uint32).copy().reshape(2500, 2)
    return {"n_contrib": n, "ranges": ranges}


def case_list():
    """name -> (scene kwargs, camera kwargs, degree, render size, grad kinds)"""
    c = {}
    c["native800_16k"] = dict(scene=dict(P=16384, seed=0, layout="shell"), cam=dict(az=0.0, el=0.0, r=2.5),
                              size=800, degree=3, grads="color")
    for v in range(4):
        c[f"crop256_16k_v{v}"] = dict(scene=dict(P=16384, seed=0, layout="shell"),
                                      cam=dict(az=90.0 * v, el=0.0, r=2.5), size=256, degree=3, grads="color")
    c["native800_16k_deg0"] = dict(scene=dict(P=16384, seed=7, layout="shell"), cam=dict(az=30.0, el=20.0, r=2.5),
                                   size=800, degree=0, grads="all")
    c["native800_2k_large"] = dict(scene=dict(P=2048, seed=11, layout="shell", log_scale=(-3.5, -2.0)),
                                   cam=dict(az=200.0, el=-15.0, r=2.5), size=800, degree=3, grads="all")
    c["crop128_1k_small"] = dict(scene=dict(P=1024, seed=5, layout="shell"), cam=dict(az=45.0, el=10.0, r=2.5),
                                 size=128, degree=3, grads="all")
    c["native800_1k_far"] = dict(scene=dict(P=1024, seed=13, layout="shell"), cam=dict(az=120.0, el=-20.0, r=6.0),
                                 size=800, degree=3, grads="all")
    return c


SMALL_CASES = ["crop128_1k_small", "native800_1k_far"]


def build_case(spec):
    sc = scenes.make_scene(**spec["scene"])
    cam = camera.orbit_camera(spec["cam"]["az"], spec["cam"]["el"], spec["cam"]["r"], spec["size"], spec["size"])
    return sc, cam


def run_case(ref, name, spec, full: bool, repeats: int = 3):
    import torch
    sc, cam = build_case(spec)
    means3D, opac, scales, rots, shs = sc.activate()
    ecam = cam if cam.width == FRAME else camera.crop_embed(cam, FRAME)
    dev = "cuda"
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    args = (t(shs), float(ecam.focal_y), t(scales), t(means3D), t(ecam.projmatrix), int(spec["degree"]), t(opac),
            t(rots), t(ecam.campos), t(ecam.viewmatrix), float(cam.focal_x))
    runs = []
    for _ in range(repeats):
        out = ref.rasterize_gaussians(*args)
        torch.cuda.synchronize()
        runs.append(out)
    R, color, depth, alpha, radii, geom, binb, img = runs[0]
    P = means3D.shape[0]
    g = carve_geom(geom.cpu().numpy(), P)
    b = carve_bin(binb.cpu().numpy(), R)
    im = carve_img(img.cpu().numpy())
    det_keys = [np.array_equal(carve_bin(r[6].cpu().numpy(), R)["keys"], b["keys"]) for r in runs[1:]]
    det_vals = [np.array_equal(carve_bin(r[6].cpu().numpy(), R)["point_list"], b["point_list"]) for r in runs[1:]]
    det_unsorted = [np.array_equal(carve_bin(r[6].cpu().numpy(), R)["unsorted_vals"], b["unsorted_vals"])
                    for r in runs[1:]]
    det_img = [torch.equal(r[1], color) for r in runs[1:]]
    rng = np.random.default_rng(1234)
    S = spec["size"]
    dLc = np.zeros((3, FRAME, FRAME), np.float32)
    dLc[:, :S, :S] = rng.normal(size=(3, S, S))
    dLd = np.zeros((1, FRAME, FRAME), np.float32)
    dLa = np.zeros((1, FRAME, FRAME), np.float32)
    if spec["grads"] == "all":
        dLd[:, :S, :S] = rng.normal(size=(1, S, S))
        dLa[:, :S, :S] = rng.normal(size=(1, S, S))
    bg = torch.ones(3, device=dev)
    empty = torch.empty(0, device=dev)
    grads = ref.rasterize_gaussians_backward(
        bg, t(means3D), radii, empty, t(scales), t(rots), 1.0, empty, t(ecam.viewmatrix), t(ecam.projmatrix),
        float(cam.tanfovx * FRAME / cam.width), float(cam.tanfovy * FRAME / cam.height), t(dLc), t(dLd), t(dLa),
        t(shs), int(spec["degree"]), t(ecam.campos), geom, R, binb, img, alpha, False)
    torch.cuda.synchronize()
    names = ["dL_dmeans2D", "dL_dcolors", "dL_dopacity", "dL_dmeans3D", "dL_dcov3D", "dL_dsh", "dL_dscales",
             "dL_drotations"]
    res = dict(P=P, R=int(R), size=S, degree=spec["degree"], radii=radii.cpu().numpy())
    if full:
        y0, y1, x0, x1 = 0, FRAME, 0, FRAME
    else:  # the tile-aligned box of non-empty pixels (everything else is background)
        nz = np.nonzero(im["n_contrib"][:S, :S])
        y0, y1 = int(nz[0].min()) // 16 * 16, (int(nz[0].max()) // 16 + 1) * 16
        x0, x1 = int(nz[1].min()) // 16 * 16, (int(nz[1].max()) // 16 + 1) * 16
    res["img_box"] = np.array([y0, y1, x0, x1])
    res["color"] = color.cpu().numpy()[:, y0:y1, x0:x1]
    res["depth_img"] = depth.cpu().numpy()[:, y0:y1, x0:x1]
    res["alpha"] = alpha.cpu().numpy()[:, y0:y1, x0:x1]
    res["n_contrib"] = im["n_contrib"][y0:y1, x0:x1]
    res["ranges"] = im["ranges"]
    for k, v in g.items():
        res["geom_" + k] = v
    for k, v in b.items():
        res["bin_" + k] = v
    for k, v in zip(names, grads):
        res[k] = v.cpu().numpy()
    # upstream gradients outside the image box meet no Gaussian and are not stored
    res["dL_dcolor_in"] = dLc[:, y0:y1, x0:x1]
    res["dL_ddepth_in"] = dLd[:, y0:y1, x0:x1]
    res["dL_dalpha_in"] = dLa[:, y0:y1, x0:x1]
    res["in_means3D"], res["in_opac"], res["in_scales"], res["in_rots"], res["in_shs"] = means3D, opac, scales, rots, shs
    res["cam_view"], res["cam_proj"], res["cam_campos"] = ecam.viewmatrix, ecam.projmatrix, ecam.campos
    res["cam_focal_x"] = np.float32(cam.focal_x)
    res["cam_tan"] = np.array([cam.tanfovx, cam.tanfovy], np.float64)
    res["determinism"] = np.array([all(det_keys), all(det_vals), all(det_unsorted), all(det_img)])
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--full", action="store_true")
    ap.add_argument("--cases", default="")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    ref = load_reference()
    allc = case_list()
    names = [n for n in a.cases.split(",") if n] or (list(allc) if a.full else SMALL_CASES)
    import torch
    info = dict(gpu=torch.cuda.get_device_name(0), torch=torch.__version__)
    print(info)
    for n in names:
        t0 = time.time()
        res = run_case(ref, n, allc[n], a.full)
        np.savez_compressed(os.path.join(a.out, n + ".npz"), **res)
        print(n, "P", res["P"], "R", res["R"], "determinism", res["determinism"].tolist(), "%.2fs" % (time.time() - t0),
              flush=True)


if __name__ == "__main__":
    main()
