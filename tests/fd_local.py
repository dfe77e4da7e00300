"""Finite differences of the rendered loss at full scene size, evaluated
locally (test infrastructure).

Perturbing one parameter of Gaussian i changes only the pixels of the tiles
its rectangle covers.  With the allocation-rectangle key emission
(compat_spill=False) a tile's list holds exactly the Gaussians whose
rectangle covers it, ordered by depth and then by index, so rendering just
the Gaussians that reach a neighbourhood of i's rectangle reproduces the
full render on that neighbourhood exactly.  The loss difference between the
+h and -h renders is then summed over the neighbourhood's pixels only.

Used by the config-2 finite-difference test to check the CUDA path's
exact-mode gradients at 500k Gaussians, where re-rendering the whole scene
per evaluation would take minutes.
"""
from __future__ import annotations

import numpy as np

import oracle

PARAM_NAMES = ("means3D", "scales", "rotations", "opacities", "shs")


def tile_grid(st):
    return (st.W + 15) // 16, (st.H + 15) // 16


def neighbourhood(base: dict, i: int, margin: int = 0):
    """Tile rectangle [x0, x1) x [y0, y1) around Gaussian i's rectangle."""
    gw, gh = tile_grid(base["settings"])
    x0, y0, x1, y1 = (int(v) for v in base["rects"][i])
    return max(0, x0 - margin), max(0, y0 - margin), min(gw, x1 + margin), min(gh, y1 + margin)


def members(base: dict, box) -> np.ndarray:
    """Gaussians in the lists of the box's tiles (sorted indices)."""
    gw, _ = tile_grid(base["settings"])
    x0, y0, x1, y1 = box
    ids = []
    for ty in range(y0, y1):
        for tx in range(x0, x1):
            s, e = base["ranges"][ty * gw + tx]
            ids.append(base["point_list"][s:e])
    return np.unique(np.concatenate(ids)) if ids else np.zeros(0, np.int64)


def box_pixels(st, box):
    x0, y0, x1, y1 = box
    return slice(16 * y0, min(st.H, 16 * y1)), slice(16 * x0, min(st.W, 16 * x1))


def box_tiles(st, box) -> np.ndarray:
    gw, _ = tile_grid(st)
    x0, y0, x1, y1 = box
    return np.array([ty * gw + tx for ty in range(y0, y1) for tx in range(x0, x1)], np.int64)


def local_render(st, params: dict, subset: np.ndarray, box, precision="f64") -> dict:
    p = {k: np.ascontiguousarray(np.asarray(v)[subset]) for k, v in params.items()}
    return oracle.forward(st, p["means3D"], p["scales"], p["rotations"], p["opacities"], p["shs"],
                          precision=precision, only_tiles=box_tiles(st, box))


def central_difference(st, params: dict, base: dict, dL_dcolor, name: str, idx: tuple, rel_h: float = 1e-3):
    """(fd, skipped_reason or None, h) for parameter params[name][idx] of
    Gaussian idx[0]."""
    i = idx[0]
    box = neighbourhood(base, i)
    sub = members(base, box)
    if i not in set(sub.tolist()):
        sub = np.union1d(sub, [i])
    k = int(np.searchsorted(sub, i))
    arr = np.asarray(params[name])
    h = rel_h * max(abs(float(arr[idx])), 1e-2)
    renders = []
    for sign in (1.0, -1.0):
        local = {kk: np.asarray(v)[sub].copy() for kk, v in params.items()}
        li = (k,) + tuple(idx[1:])
        local[name][li] = np.float32(float(arr[idx]) + sign * h)
        renders.append((oracle.forward(st, local["means3D"], local["scales"], local["rotations"],
                                       local["opacities"], local["shs"], precision="f64",
                                       only_tiles=box_tiles(st, box)), float(local[name][li])))
    (fp, vp), (fm, vm) = renders
    hh = (vp - vm) / 2.0
    # the perturbed Gaussian must stay inside the neighbourhood
    for f in (fp, fm):
        x0, y0, x1, y1 = (int(v) for v in f["rects"][k])
        if f["radii"][k] > 0 and (x0 < box[0] or y0 < box[1] or x1 > box[2] or y1 > box[3]):
            return None, "left the neighbourhood", hh
    rows, cols = box_pixels(st, box)
    tiles = box_tiles(st, box)
    lists = lambda f: [f["point_list"][f["ranges"][t][0]:f["ranges"][t][1]] for t in tiles]
    if not (np.array_equal(fp["blend_signature"][rows, cols], fm["blend_signature"][rows, cols])
            and all(np.array_equal(a, b) for a, b in zip(lists(fp), lists(fm)))):
        return None, "blend decision changed", hh
    g = np.asarray(dL_dcolor, np.float64)[:, rows, cols]
    dl = float(np.sum((np.asarray(fp["color"], np.float64)[:, rows, cols] -
                       np.asarray(fm["color"], np.float64)[:, rows, cols]) * g))
    return dl / (2.0 * hh), None, hh
