"""Pin the CPU oracle to the reference extension's own outputs.

The fixtures in tests/golden/ were written by tests/golden/make_golden.py,
which runs the reference extension (built from the reference sources) on a
B200.  Checked on the CPU:

* per-Gaussian fields bit-exact (depth, screen position, 3-D covariance,
  conic, colour, clamp flags, radius, tiles touched, offsets);
* the unsorted key/id arrays: bit-exact at single-writer slots; at slots the
  reference's racing emission writes several times, its entry is one of the
  candidate writes;
* the oracle's stable sort of the reference's unsorted arrays, and tile
  ranges from its sorted keys, reproduce the reference bit-exactly;
* blending the reference's sorted lists: contributor counts exact except at
  pixels within 1e-5 of a threshold (C-library vs device exp), images within
  1e-5 + 1e-4|x|;
* the reference-formula backward on the same state: gradients within
  parity.grad_check bounds and 1e-4 norm-relative.
"""
import ctypes
import glob
import os

import numpy as np
import pytest

import oracle
import parity

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
FRAME = 800

if not FIXTURES:
    pytest.skip("no golden fixtures", allow_module_level=True)


def _settings(d):
    st = oracle.RasterSettings(W=FRAME, H=FRAME, viewmatrix=d["cam_view"], projmatrix=d["cam_proj"],
                               campos=d["cam_campos"], focal_x=float(d["cam_focal_x"]), degree=int(d["degree"]))
    return st


@pytest.fixture(scope="module", params=FIXTURES, ids=[os.path.basename(f) for f in FIXTURES])
def case(request):
    d = dict(np.load(request.param))
    st = _settings(d)
    f = oracle.forward(st, d["in_means3D"], d["in_scales"], d["in_rots"], d["in_opac"], d["in_shs"])
    return d, st, f


def test_geometry_bit_exact(case):
    d, st, f = case
    for k in ("depth", "means2D", "cov3D", "conic_opac", "rgb", "tiles", "offsets"):
        assert parity.bit_mismatch(np.asarray(f[k], np.float32) if f[k].dtype.kind == "f" else f[k],
                                   d["geom_" + k]) == 0, k
    assert parity.bit_mismatch(f["clamped"], d["geom_clamped"]) == 0
    assert parity.bit_mismatch(f["radii"], d["radii"]) == 0
    assert f["num_rendered"] == int(d["R"])


def test_key_emission(case):
    d, st, f = case
    uk, uv = d["bin_unsorted_keys"], d["bin_unsorted_vals"]
    diff = (uk != f["unsorted_keys"]) | (uv != f["unsorted_vals"])
    single = f["candidates"] <= 1
    assert int((diff & single).sum()) == 0
    start = np.concatenate([[0], f["offsets"][:-1]]).astype(np.int64)
    for p in np.nonzero(diff & ~single)[0]:
        owner = np.searchsorted(start, p, side="right") - 1
        lo = max(0, owner - 64)
        assert lo <= uv[p] <= owner, (p, uv[p], owner)


def test_sort_and_ranges_replay(case):
    d, st, f = case
    k = d["bin_unsorted_keys"].copy()
    v = d["bin_unsorted_vals"].copy()
    oracle.lib().orc_sort_pairs_u64(oracle._p(k), oracle._p(v), ctypes.c_longlong(len(k)))
    assert np.array_equal(k, d["bin_keys"]) and np.array_equal(v, d["bin_point_list"])
    ranges = np.zeros((2500, 2), np.uint32)
    oracle.lib().orc_tile_ranges(oracle._p(d["bin_keys"]), ctypes.c_longlong(len(k)), oracle._p(ranges),
                                 ctypes.c_int(2500))
    assert np.array_equal(ranges, d["ranges"])


def _replay(d, st, f):
    b = oracle.blend(st, f, d["ranges"], d["bin_point_list"])
    y0, y1, x0, x1 = d["img_box"]
    return b, (slice(y0, y1), slice(x0, x1))


def test_blend_replay(case):
    d, st, f = case
    b, (ys, xs) = _replay(d, st, f)
    nc = parity.ncontrib_check(b["n_contrib"][ys, xs], d["n_contrib"], b["blend_margin"][ys, xs])
    assert nc["n_unexplained"] == 0, nc
    keep = ~nc["mask"] & (b["blend_margin"][ys, xs] >= 1e-5)
    for k in ("color", "alpha", "depth_img"):
        e = parity.err_stats(b[k][:, ys, xs][:, keep], d[k][:, keep])
        assert e["n_bad"] == 0, (k, e)


def test_backward_replay(case):
    d, st, f = case
    b, (ys, xs) = _replay(d, st, f)
    alpha = np.zeros((1, FRAME, FRAME), np.float32)
    alpha[:, ys, xs] = d["alpha"]
    nc = np.zeros((FRAME, FRAME), np.uint32)
    nc[ys, xs] = d["n_contrib"]
    fwd = dict(f, ranges=d["ranges"], point_list=d["bin_point_list"], alpha=alpha, n_contrib=nc,
               num_rendered=int(d["R"]))
    g = {}
    for k, shape in (("dL_dcolor_in", 3), ("dL_ddepth_in", 1), ("dL_dalpha_in", 1)):
        full = np.zeros((shape, FRAME, FRAME), np.float32)
        full[:, ys, xs] = d[k]
        g[k] = full
    S = int(d["size"])
    tan = np.asarray(d["cam_tan"]) * FRAME / S
    out = oracle.backward(fwd, g["dL_dcolor_in"], g["dL_ddepth_in"], g["dL_dalpha_in"], tan_fovx=tan[0],
                          tan_fovy=tan[1])
    for k in parity.GRAD_NAMES:
        c = parity.grad_check(out[k], d[k], row_rtol=0.0, abs_sum=out.get("abs_" + k))
        print(k, {x: c[x] for x in ("norm_rel", "n_bad", "n_elem_strict", "n")})
        assert c["norm_rel"] <= 1e-4 and c["n_bad"] == 0, (k, c)
