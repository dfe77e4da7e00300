"""CUDA rasterizer vs the CPU oracle on the same seeded inputs.

Bit-exact: every per-Gaussian field (depth, screen position, 3-D
covariance, conic, colour, radius, tiles touched, offsets), the instance
count, the sorted 64-bit keys, the sorted Gaussian ids and the per-tile
ranges.  Contributor counts: exact except at pixels whose blend decisions
lie within 1e-5 (relative) of a threshold, where the device and C-library
exp may round differently.  Images and gradients: |a-b| <= 1e-5 + 1e-4|b|
(gradients with the fp32 accumulation-order term of parity.grad_check) and
norm-relative error <= 1e-4 per result.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

import oracle  # noqa: E402
import parity  # noqa: E402
import gpu_helpers as gh  # noqa: E402
from word2world_b200 import _C, camera, scenes  # noqa: E402


def _setup(P=4096, seed=0, layout="shell", size=128, az=30.0, el=10.0, degree=3, log_scale=(-5.0, -3.0),
           M=16, W=None, H=None, radius=2.5):
    sc = scenes.make_scene(P, seed=seed, layout=layout, log_scale=log_scale)
    m, o, s, q, sh = sc.activate()
    sh = np.ascontiguousarray(sh[:, :M])
    W = size if W is None else W
    H = size if H is None else H
    cam = camera.orbit_camera(az, el, radius, W, H)
    return (m, o, s, q, sh), cam


def _orc(arrays, cam, degree=3, compat_spill=True, bg=(1.0, 1.0, 1.0)):
    m, o, s, q, sh = arrays
    st = oracle.RasterSettings.from_camera(cam, degree=degree, bg=bg, compat_spill=compat_spill)
    return oracle.forward(st, m, s, q, o, sh)


def _check_forward(mine, orc, img_tol=True):
    gm = parity.geometry_mismatches(mine, orc, visible=orc["visible"].astype(bool))
    assert all(v == 0 for v in gm.values()), gm
    assert mine["num_rendered"] == orc["num_rendered"]
    assert parity.bit_mismatch(mine["keys"], orc["keys"]) == 0
    assert parity.bit_mismatch(mine["point_list"], orc["point_list"]) == 0
    assert parity.bit_mismatch(mine["ranges"], orc["ranges"]) == 0
    nc = parity.ncontrib_check(mine["n_contrib"], orc["n_contrib"], orc["blend_margin"])
    assert nc["n_unexplained"] == 0, nc
    assert nc["n_diff"] <= max(2, nc["n"] // 10000), nc
    if img_tol:
        keep = ~nc["mask"] & (np.asarray(orc["blend_margin"]) >= 1e-5)
        for k in ("color", "alpha", "depth_img"):
            a, b = mine[k], orc[k]
            e = parity.err_stats(a[:, keep], b[:, keep])
            assert e["n_bad"] == 0, (k, e)
    return nc


@pytest.mark.parametrize("view", [0, 1, 2, 3])
def test_forward_16k_256(view):
    """16,384 Gaussians, 4 orbit views at 256x256, SH degree 3."""
    sc = scenes.scene_16k(0)
    arrays = sc.activate()
    cam = camera.orbit_views(4, 2.5, 256, 256)[view]
    mine = gh.forward(arrays, cam)
    orc = _orc(arrays, cam)
    _check_forward(mine, orc)


@pytest.mark.parametrize("compat_spill", [True, False])
@pytest.mark.parametrize("degree,M", [(0, 1), (0, 16), (1, 4), (2, 9), (3, 16)])
def test_forward_degrees_and_spill(degree, M, compat_spill):
    arrays, cam = _setup(P=3000, seed=degree + 10 * M, size=160, degree=degree, M=M)
    mine = gh.forward(arrays, cam, degree=degree, compat_spill=compat_spill)
    orc = _orc(arrays, cam, degree=degree, compat_spill=compat_spill)
    _check_forward(mine, orc)


@pytest.mark.parametrize("W,H", [(250, 130), (17, 33), (1, 1), (512, 96)])
def test_forward_ragged_sizes(W, H):
    # far enough that no Gaussian reaches the inscribed-circle clamp, whose
    # approximate reciprocal square root is outside the oracle's bit contract
    arrays, cam = _setup(P=2500, seed=3, W=W, H=H, log_scale=(-4.5, -2.5), radius=8.0)
    mine = gh.forward(arrays, cam)
    orc = _orc(arrays, cam)
    assert not orc["clamp_hit"].any()
    _check_forward(mine, orc)


def test_forward_circle_clamp():
    """Gaussians outside the inscribed circle of a narrow image are pulled onto
    it with the reference's rsqrtf: geometry that does not depend on the clamp
    stays bit-exact, the conic agrees to a few ulps."""
    arrays, cam = _setup(P=2500, seed=3, W=17, H=33, log_scale=(-4.5, -2.5))
    mine = gh.forward(arrays, cam)
    orc = _orc(arrays, cam)
    hit = orc["clamp_hit"].astype(bool)
    vis = orc["visible"].astype(bool)
    assert hit.any()
    for k in ("depth", "means2D", "cov3D"):
        assert parity.bit_mismatch(mine[k][vis], np.asarray(orc[k], np.float32)[vis]) == 0, k
    ok = vis & ~hit
    assert parity.bit_mismatch(mine["conic_opac"][ok], orc["conic_opac"][ok]) == 0
    e = parity.err_stats(mine["conic_opac"][hit & vis], orc["conic_opac"][hit & vis], atol=0, rtol=1e-5)
    assert e["n_bad"] == 0, e


def test_forward_background_and_large_gaussians():
    arrays, cam = _setup(P=1500, seed=4, size=200, log_scale=(-3.0, -1.5))
    bg = (0.2, 0.5, 0.9)
    mine = gh.forward(arrays, cam, bg=bg)
    orc = _orc(arrays, cam, bg=bg)
    _check_forward(mine, orc)


def test_forward_empty_and_culled():
    # P = 0
    arrays, cam = _setup(P=0, size=64)
    mine = gh.forward(arrays, cam)
    assert mine["num_rendered"] == 0
    assert np.allclose(mine["color"], 1.0) and np.all(mine["n_contrib"] == 0)
    # every Gaussian behind the near test (view z <= 1): all culled
    arrays, cam = _setup(P=500, size=64)
    m = arrays[0].copy()
    m[:] = np.asarray(cam.campos, np.float32) * -1.0  # at the camera centre
    arrays = (m,) + arrays[1:]
    mine = gh.forward(arrays, cam)
    orc = _orc(arrays, cam)
    assert mine["num_rendered"] == 0 and orc["num_rendered"] == 0
    assert np.all(mine["radii"] == 0)
    assert np.allclose(mine["color"], 1.0)
    # one Gaussian
    arrays, cam = _setup(P=1, size=64, seed=9)
    _check_forward(gh.forward(arrays, cam), _orc(arrays, cam))


def _grads(arrays, cam, mode, degree=3, seed=1, with_depth_alpha=True):
    H, W = cam.height, cam.width
    rng = np.random.default_rng(seed)
    dLc = rng.normal(size=(3, H, W)).astype(np.float32)
    dLd = rng.normal(size=(1, H, W)).astype(np.float32) if with_depth_alpha else None
    dLa = rng.normal(size=(1, H, W)).astype(np.float32) if with_depth_alpha else None
    mine_f = gh.forward(arrays, cam, degree=degree)
    mine = gh.backward(mine_f, arrays, cam, dLc, dLd, dLa, degree=degree, grad_mode=0 if mode == "reference" else 1)
    orc_f = _orc(arrays, cam, degree=degree)
    # The reference-formula backward starts from T_final = 1 - alpha, which
    # turns a 1-ulp alpha difference (device vs C-library exp) of a nearly
    # opaque pixel into a 1e-4-relative change; give the oracle this
    # implementation's alpha image so the comparison isolates the gradients.
    orc_f = dict(orc_f, alpha=mine_f["alpha"])
    orc = oracle.backward(orc_f, dLc, dLd, dLa, mode=mode)
    return mine, orc


@pytest.mark.parametrize("mode", ["reference", "exact"])
@pytest.mark.parametrize("degree", [0, 3])
def test_backward_vs_oracle(mode, degree):
    """Reference mode: the elementwise contract with the accumulation-order
    term.  Exact mode (this build's own derivative, validated by finite
    differences in test_gpu_fd.py and test_gpu_config2.py): its oracle keeps
    no sums of |per-pair terms|, so per result the norm-relative error only,
    with the elements outside the plain 1e-5 + 1e-4 |b| bound reported."""
    arrays, cam = _setup(P=4096, seed=21, size=192, degree=degree)
    mine, orc = _grads(arrays, cam, mode, degree=degree)
    report = {}
    for k in parity.GRAD_NAMES:
        c = parity.grad_check(mine[k], orc[k], abs_sum=orc.get("abs_" + k))
        report[k] = c
        assert c["norm_rel"] <= 1e-4, (k, c)
        if mode == "reference":
            assert c["n_bad"] == 0, (k, c)
    print({k: (f"{v['norm_rel']:.2e}", v["n_elem_strict"]) for k, v in report.items()})


def test_backward_16k_256_reference_mode():
    sc = scenes.scene_16k(0)
    arrays = sc.activate()
    cam = camera.orbit_views(4, 2.5, 256, 256)[0]
    mine, orc = _grads(arrays, cam, "reference", with_depth_alpha=False)
    for k in parity.GRAD_NAMES:
        c = parity.grad_check(mine[k], orc[k], abs_sum=orc.get("abs_" + k))
        assert c["norm_rel"] <= 1e-4 and c["n_bad"] == 0, (k, c)


def test_deterministic_forward():
    arrays, cam = _setup(P=8000, seed=5, size=256)
    a = gh.forward(arrays, cam)
    b = gh.forward(arrays, cam)
    for k in ("keys", "point_list", "ranges", "n_contrib", "color", "alpha"):
        assert parity.bit_mismatch(a[k], b[k]) == 0, k


BIN_CASES = {
    "16k_256_v0": dict(P=16384, seed=0, layout="shell", size=256, az=0.0, el=0.0),
    "3k_160_large": dict(P=3000, seed=30, layout="shell", size=160, log_scale=(-4.0, -2.0)),
    "ragged_250x130": dict(P=2500, seed=3, W=250, H=130, log_scale=(-4.5, -2.5), radius=8.0),
    "tiny_17x33": dict(P=2500, seed=3, W=17, H=33, log_scale=(-4.5, -2.5), radius=8.0),
    "one": dict(P=1, seed=9, size=64),
}


@pytest.mark.parametrize("compat_spill", [True, False])
@pytest.mark.parametrize("case", list(BIN_CASES))
def test_binning_paths_agree(case, compat_spill):
    """The two ways of building the sorted list -- key emission + radix sort,
    and binning from the depth-ordered Gaussians (the "binning" tuning knob)
    -- give bit-identical keys, lists, ranges, contributor counts and images,
    the oracle's, and gradients equal up to atomic order."""
    spec = dict(BIN_CASES[case])
    arrays, cam = _setup(**spec)
    rng = np.random.default_rng(4)
    g = rng.normal(size=(3, cam.height, cam.width)).astype(np.float32)
    out = {}
    for path in (0, 1):
        with gh.tuned(binning=path):
            f = gh.forward(arrays, cam, compat_spill=compat_spill)
            b = gh.backward(f, arrays, cam, g, grad_mode=0)
        out[path] = (f, b)
    (f0, b0), (f1, b1) = out[0], out[1]
    for k in ("keys", "point_list", "ranges", "n_contrib", "color", "alpha", "depth_img"):
        assert parity.bit_mismatch(f0[k], f1[k]) == 0, k
    orc = _orc(arrays, cam, compat_spill=compat_spill)
    assert parity.bit_mismatch(f1["keys"], orc["keys"]) == 0
    assert parity.bit_mismatch(f1["point_list"], orc["point_list"]) == 0
    assert parity.bit_mismatch(f1["ranges"], orc["ranges"]) == 0
    for k in parity.GRAD_NAMES:
        c = parity.grad_check(b1[k], b0[k], row_rtol=parity.SAME_IMPL_ROW_RTOL)
        assert c["norm_rel"] <= 1e-5 and c["n_bad"] == 0, (k, c)



QUEUE_CASES = dict(BIN_CASES, heavy_40k_512=dict(P=40000, seed=12, layout="ball", size=512))


@pytest.mark.parametrize("warps", [4, 8])
@pytest.mark.parametrize("case", list(QUEUE_CASES))
def test_queue_blend_agrees(case, warps):
    """The persistent blend fed by the device tile queue and TMA row gathers
    (the "blend_queue" tuning knob) gives bit-identical images, contributor
    counts and block masks (hence backward gradients) to the per-tile blend."""
    spec = dict(QUEUE_CASES[case])
    arrays, cam = _setup(**spec)
    rng = np.random.default_rng(6)
    g = rng.normal(size=(3, cam.height, cam.width)).astype(np.float32)
    out = {}
    for queue in (0, 1):
        with gh.tuned(blend_warps=warps, blend_queue=queue):
            f = gh.forward(arrays, cam)
            b = gh.backward(f, arrays, cam, g, grad_mode=0)
            _C.check_device_errors()  # no bounded wait of the queue ran out
        out[queue] = (f, b)
    (f0, b0), (f1, b1) = out[0], out[1]
    for k in ("point_list", "ranges", "n_contrib", "color", "alpha", "depth_img"):
        assert parity.bit_mismatch(f0[k], f1[k]) == 0, k
    for k in parity.GRAD_NAMES:
        c = parity.grad_check(b1[k], b0[k], row_rtol=parity.SAME_IMPL_ROW_RTOL)
        assert c["norm_rel"] <= 1e-5 and c["n_bad"] == 0, (k, c)
