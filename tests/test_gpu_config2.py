"""Parity at the benchmarked configuration: 500,000 Gaussians uniformly in a
radius-0.6 ball, SH degree 3, the 4 orbit views at 512x512, the reference's
key emission (compat_spill) -- the workload bench.py measures.

Per view, the CUDA path (its own forward, then its backward from that
forward's state) against the oracle (fp32):

* bit-exact: every per-Gaussian field, the instance count, the sorted 64-bit
  keys and Gaussian ids, the tile ranges -- by the default radix path and by
  the depth-ordered binning alike;
* contributor counts exact except at pixels whose blend decisions lie
  within 1e-5 (relative) of a threshold, where the device exp and the C
  library's may round differently;
* images: |a - b| <= 1e-5 + 1e-4 |b| at every other pixel;
* gradients: every result's error reported (norm-relative, worst absolute,
  n_elem_strict = elements outside 1e-5 + 1e-4 |b|) end to end, and the
  strict contract -- 1e-5 + 1e-4 |b| plus only the fp32 accumulation-order
  term 64 ulp x sum |per-pair terms| -- on the isolated backward (see
  test_config2_backward).

Then the fp64 re-evaluation (errors reported per result, two ways), and
central finite differences (h = 1e-3) of the fp64 forward on 256 seeded
parameters against the exact-mode gradients, evaluated locally around each
perturbed Gaussian (tests/fd_local.py).
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

import fd_local  # noqa: E402
import gpu_helpers as gh  # noqa: E402
import oracle  # noqa: E402
import parity  # noqa: E402
from word2world_b200 import camera, scenes  # noqa: E402

S = 512
_CACHE = {}


def _cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


@pytest.fixture(scope="module")
def workload():
    oracle.set_threads(_cores())  # results do not depend on it (the backward's double sums only in order)
    arrays = scenes.scene_500k(0).activate()
    cams = camera.orbit_views(4, 2.5, S, S)
    grads = scenes.upstream_grads(4, S, S, seed=1)
    yield arrays, cams, grads
    oracle.set_threads(1)
    _CACHE.clear()


def _view(workload, v):
    if v in _CACHE:
        return _CACHE[v]
    arrays, cams, grads = workload
    m, o, s, q, sh = arrays
    cam = cams[v]
    mine = gh.forward(arrays, cam)
    mine_b = gh.backward(mine, arrays, cam, grads[v], grad_mode=0)
    st = oracle.RasterSettings.from_camera(cam)
    orc = oracle.forward(st, m, s, q, o, sh)
    orc_b = oracle.backward(orc, grads[v], mode="reference")
    _CACHE[v] = (mine, mine_b, orc, orc_b)
    return _CACHE[v]


def _forward_state(workload, v):
    """This implementation's forward of view v (with its device state)."""
    return _view(workload, v)[0]


@pytest.mark.parametrize("view", [0, 1, 2, 3])
def test_config2_forward(workload, view):
    mine, _, orc, _ = _view(workload, view)
    gm = parity.geometry_mismatches(mine, orc, visible=orc["visible"].astype(bool))
    assert all(v == 0 for v in gm.values()), gm
    assert mine["num_rendered"] == orc["num_rendered"]
    assert parity.bit_mismatch(mine["keys"], orc["keys"]) == 0
    assert parity.bit_mismatch(mine["point_list"], orc["point_list"]) == 0
    assert parity.bit_mismatch(mine["ranges"], orc["ranges"]) == 0
    nc = parity.ncontrib_check(mine["n_contrib"], orc["n_contrib"], orc["blend_margin"])
    assert nc["n_unexplained"] == 0, nc
    keep = ~nc["mask"] & (np.asarray(orc["blend_margin"]) >= 1e-5)
    report = {"R": mine["num_rendered"], "ncontrib_diff": nc["n_diff"], "pixels_in_band": int((~keep).sum())}
    for k in ("color", "alpha", "depth_img"):
        e = parity.err_stats(mine[k][:, keep], orc[k][:, keep])
        whole = parity.err_stats(mine[k], orc[k])
        report[k] = {"max_abs": e["max_abs"], "norm_rel": whole["norm_rel"], "bits_equal":
                     1.0 - parity.bit_mismatch(mine[k], orc[k]) / mine[k].size}
        assert e["n_bad"] == 0, (k, e)
    print(f"view {view} forward:", report)


@pytest.mark.parametrize("view", [0, 2])
def test_config2_binning_path(workload, view):
    """The depth-ordered binning (the "binning" tuning knob) builds the same
    sorted list at this size: keys, ids, ranges and images bit-identical to
    the radix path's, which the forward test pins to the oracle."""
    arrays, cams, _ = workload
    mine = _view(workload, view)[0]
    with gh.tuned(binning=1):
        alt = gh.forward(arrays, cams[view])
    for k in ("keys", "point_list", "ranges", "n_contrib", "color", "alpha", "depth_img"):
        assert parity.bit_mismatch(alt[k], mine[k]) == 0, k


@pytest.mark.parametrize("view", [0, 1, 2, 3])
def test_config2_backward(workload, view):
    """Two comparisons per result.

    End to end (each side from its own forward): the reference backward
    restarts the transmittance from T_final = 1 - alpha (backward.cu:565),
    so the last-bit differences of the alpha image (device vs C-library exp:
    about an eighth of the pixels differ in their last bits, by at most
    6e-7) come back amplified by up to 1 / T_final (1e4 at the 1e-4
    termination threshold) in the gradients of nearly opaque pixels.  These
    errors are reported and bounded at 1e-3 norm-relative.

    Isolated: the oracle's backward on this implementation's alpha image,
    both sides with the upstream gradient zeroed at the pixels whose
    backward recomputes a pair's alpha within 1e-5 (relative) of the 1/255
    skip threshold, or whose forward decisions sit that close to theirs
    (there the device exp and the C library's may decide differently, as in
    the forward's contributor counts).  Strict contract: 1e-5 + 1e-4 |b| plus
    the accumulation-order term per element, 1e-4 norm-relative per result."""
    arrays, cams, grads = workload
    mine, mine_b, orc, orc_b = _view(workload, view)
    e2e, iso = {}, {}
    for k in parity.GRAD_NAMES:
        c = parity.grad_check(mine_b[k], orc_b[k], row_rtol=0.0, abs_sum=orc_b.get("abs_" + k))
        e2e[k] = {x: c[x] for x in ("norm_rel", "max_abs", "n_elem_strict", "n")}
    shared = oracle.backward(dict(orc, alpha=mine["alpha"]), grads[view], mode="reference")
    band = (np.asarray(shared["backward_margin"]) < 1e-5) | (np.asarray(orc["blend_margin"]) < 1e-5)
    g = np.where(band[None], 0.0, grads[view]).astype(np.float32)
    mine_m = gh.backward(_forward_state(workload, view), arrays, cams[view], g, grad_mode=0)
    orc_m = oracle.backward(dict(orc, alpha=mine["alpha"]), g, mode="reference")
    for k in parity.GRAD_NAMES:
        c = parity.grad_check(mine_m[k], orc_m[k], row_rtol=0.0, abs_sum=orc_m.get("abs_" + k))
        iso[k] = {x: c[x] for x in ("norm_rel", "max_abs", "n_elem_strict", "n_bad", "n")}
    print(f"view {view} backward vs oracle fp32, end to end:", e2e)
    print(f"view {view} backward vs oracle fp32, on this implementation's alpha, "
          f"{int(band.sum())} threshold pixels without upstream gradient:", iso)
    for k in parity.GRAD_NAMES:
        assert e2e[k]["norm_rel"] <= 1e-3, (k, e2e[k])
        assert iso[k]["norm_rel"] <= 1e-4, (k, iso[k])
        assert iso[k]["n_bad"] == 0, (k, iso[k])


@pytest.mark.parametrize("view", [0, 2])
def test_config2_fp64_reevaluation(workload, view):
    """The fp64 re-evaluation, two ways.  (a) The whole path in double: its
    blend makes a few different decisions (an alpha or a transmittance on the
    other side of a threshold), and its own alpha image restarts the
    reference backward's transmittance chain, so image and gradient errors
    are reported per result with loose bounds.  (b) The backward in double on
    this implementation's decisions (its sorted list, contributor counts and
    alpha image): the arithmetic precision of the reference's backward in
    fp32, which restarts the transmittance from T_final and divides it by
    (1 - alpha) once per entry walked -- each alpha's rounding enters at up to
    1 / (1 - alpha) = 100 times, over hundreds of entries -- measured at
    0.6-3e-4 norm-relative per result and bounded at 1e-3."""
    arrays, cams, grads = workload
    mine, mine_b, _, _ = _view(workload, view)
    m, o, s, q, sh = arrays
    st = oracle.RasterSettings.from_camera(cams[view])
    f64 = oracle.forward(st, m, s, q, o, sh, precision="f64")
    b64 = oracle.backward(f64, grads[view], mode="reference", error_bounds=False)
    nc_diff = int(np.count_nonzero(np.asarray(f64["n_contrib"]) != np.asarray(mine["n_contrib"])))
    full = {"same_point_list": bool(np.array_equal(f64["point_list"], mine["point_list"])),
            "pixels_with_other_decisions": nc_diff}
    for k in ("color", "alpha", "depth_img"):
        e = parity.err_stats(mine[k], f64[k])
        full[k] = {"norm_rel": e["norm_rel"], "max_abs": e["max_abs"], "n_outside_1e-5+1e-4": e["n_bad"]}
    for k in parity.GRAD_NAMES:
        c = parity.grad_check(mine_b[k], b64[k], row_rtol=0.0)
        full[k] = {x: c[x] for x in ("norm_rel", "max_abs", "n_elem_strict", "n")}
    same = dict(f64, point_list=mine["point_list"], ranges=mine["ranges"], n_contrib=mine["n_contrib"],
                alpha=np.asarray(mine["alpha"], np.float64))
    b64s = oracle.backward(same, grads[view], mode="reference", error_bounds=False)
    shared = {}
    for k in parity.GRAD_NAMES:
        c = parity.grad_check(mine_b[k], b64s[k], row_rtol=0.0)
        shared[k] = {x: c[x] for x in ("norm_rel", "max_abs", "n_elem_strict", "n")}
    print(f"view {view} vs fp64, whole path in double:", full)
    print(f"view {view} vs fp64 backward on this implementation's decisions:", shared)
    for k in ("color", "alpha", "depth_img"):
        assert full[k]["norm_rel"] <= 1e-3, (k, full[k])
    for k in parity.GRAD_NAMES:
        assert full[k]["norm_rel"] <= 1e-1, (k, full[k])
        assert shared[k]["norm_rel"] <= 1e-3, (k, shared[k])


def test_config2_finite_differences(workload):
    """Exact-mode gradients of view 0 (allocation-rectangle key emission, so
    each tile's list is exactly the Gaussians whose rectangle covers it)
    against central differences of the fp64 forward, on 256 seeded
    (Gaussian, component) draws among the Gaussians that reach the image;
    draws whose +-h perturbation changes a blend decision are skipped and
    counted."""
    arrays, cams, grads = workload
    m, o, s, q, sh = arrays
    cam, g = cams[0], grads[0]
    mine = gh.forward(arrays, cam, compat_spill=False)
    b = gh.backward(mine, arrays, cam, g, grad_mode=1)
    an_all = dict(means3D=b["dL_dmeans3D"], scales=b["dL_dscales"], rotations=b["dL_drotations"],
                  opacities=b["dL_dopacity"], shs=b["dL_dsh"])
    gmax = {k: float(np.abs(v).max()) for k, v in an_all.items()}
    params = dict(means3D=m, scales=s, rotations=q, opacities=o, shs=sh)
    st = oracle.RasterSettings.from_camera(cam, compat_spill=False)
    base = oracle.forward(st, m, s, q, o, sh, precision="f64")
    dop = np.abs(b["dL_dopacity"][:, 0])
    reach = np.nonzero(dop > 1e-4 * dop.max())[0]
    rng = np.random.default_rng(256)
    checked, skipped, worst, errs = 0, 0, 0.0, []
    for k in range(256):
        name = fd_local.PARAM_NAMES[k % len(fd_local.PARAM_NAMES)]
        arr = params[name]
        i = int(rng.choice(reach))
        idx = (i,) + tuple(int(rng.integers(0, d)) for d in arr.shape[1:])
        fd, why, _ = fd_local.central_difference(st, params, base, g, name, idx)
        if why is not None:
            skipped += 1
            continue
        an = float(np.asarray(an_all[name]).reshape(arr.shape)[idx])
        err = abs(fd - an) / max(abs(fd), 1e-3 * gmax[name], 1e-12)
        errs.append((err, name, idx, fd, an))
        checked += 1
    e = np.array([x[0] for x in errs])
    worst = max(errs)
    print(f"config-2 finite differences: {checked} checked, {skipped} skipped (a blend decision changed); "
          f"relative error median {np.median(e):.2e}, 90th percentile {np.percentile(e, 90):.2e}, "
          f"worst {worst[0]:.2e} ({worst[1]} {worst[2]}: fd {worst[3]:.6g}, gradient {worst[4]:.6g})")
    outliers = sorted(x for x in errs if x[0] > 1e-2)
    print("draws above 1e-2:", [(f"{x[0]:.2e}", x[1], x[2]) for x in outliers])
    assert checked >= 64, (checked, skipped)
    # the fp32 gradient sums thousands of per-pixel terms per Gaussian here;
    # a draw whose difference quotient is small against those terms (or whose
    # perturbation moves a decision the per-pixel signature does not track)
    # can miss by more; the bulk must agree closely
    assert np.median(e) <= 2e-3 and np.mean(e <= 1e-2) >= 0.95, (np.median(e), outliers)
