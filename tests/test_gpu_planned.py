"""The planned forward (the sort and blend launched before the instance count
is read back, into a binning state sized from earlier views of the same image
size) against the exact plan: the same instance list, tile ranges, images and
contributor counts bit for bit, gradients equal up to float atomic order --
when the plan is wider than the view needs, and when the view does not fit it
and is rendered again with the exact plan."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

import gpu_helpers as gh  # noqa: E402
import parity  # noqa: E402
from word2world_b200 import _C, camera, scenes  # noqa: E402

FIELDS = ("color", "depth_img", "alpha", "radii", "n_contrib", "ranges", "T_final", "tile_max", "keys", "point_list")


def _run(arrays, cam, planned, grad):
    with gh.tuned(planned_forward=planned):
        f = gh.forward(arrays, cam)
        g = gh.backward(f, arrays, cam, grad)
    torch.cuda.synchronize()
    return f, g


def _assert_same(f, fe, g, ge, what):
    assert f["num_rendered"] == fe["num_rendered"], what
    for k in FIELDS:
        assert parity.bit_mismatch(np.asarray(f[k]), np.asarray(fe[k])) == 0, (what, k)
    for k in ge:
        chk = parity.grad_check(g[k], ge[k], row_rtol=parity.SAME_IMPL_ROW_RTOL)
        assert chk["norm_rel"] <= 1e-5 and chk["n_bad"] == 0, (what, k, chk)


def _scene(P, seed):
    return scenes.make_scene(P, seed=seed, layout="ball").activate()


def _grad(H, W, seed):
    return np.random.default_rng(seed).normal(size=(3, H, W)).astype(np.float32)


def test_planned_forward_matches_exact():
    arrays = _scene(12000, 21)
    cam = camera.orbit_camera(30.0, 10.0, 2.5, 256, 256)
    grad = _grad(256, 256, 1)
    fe, ge = _run(arrays, cam, 0, grad)  # the exact plan
    f1, g1 = _run(arrays, cam, 1, grad)  # the shape's first planned-mode render: exact, sets the plan
    assert f1["layout_count"] == f1["num_rendered"]
    _assert_same(f1, fe, g1, ge, "first")
    for k in range(2):  # later renders launch the whole forward before reading R back
        f2, g2 = _run(arrays, cam, 1, grad)
        assert f2["layout_count"] > f2["num_rendered"], "the planned path did not run"
        _assert_same(f2, fe, g2, ge, f"planned {k}")


def test_planned_forward_with_a_wider_plan():
    """A plan from a nearer view: more capacity and more key depth bits than
    the far view needs; the extra bits are the depths' common high bits, so
    the order is the exact plan's."""
    arrays = _scene(12001, 22)
    near = camera.orbit_camera(0.0, 0.0, 1.6, 512, 512)
    far = camera.orbit_camera(0.0, 0.0, 8.0, 512, 512)
    grad = _grad(512, 512, 2)
    _run(arrays, near, 1, grad)
    ff, gf = _run(arrays, far, 1, grad)
    fe, ge = _run(arrays, far, 0, grad)
    assert ff["layout_count"] > ff["num_rendered"], "the planned path did not run"
    _assert_same(ff, fe, gf, ge, "far after near")


def test_planned_forward_falls_back_when_the_view_does_not_fit():
    arrays = _scene(30000, 23)
    near = camera.orbit_camera(0.0, 0.0, 1.6, 512, 512)
    far = camera.orbit_camera(0.0, 0.0, 8.0, 512, 512)
    grad = _grad(512, 512, 3)
    fe, ge = _run(arrays, near, 0, grad)
    ffar, _ = _run(arrays, far, 0, grad)
    lib_capacity = _C.planned_capacity(ffar["num_rendered"])
    assert fe["num_rendered"] > lib_capacity, "the near view must not fit a plan made from the far view"
    _run(arrays, far, 1, grad)  # the plan: the far view's count and depth bits
    fn, gn = _run(arrays, near, 1, grad)  # does not fit: rendered again with the exact plan
    assert fn["layout_count"] == fn["num_rendered"]
    _assert_same(fn, fe, gn, ge, "fallback")
    f3, g3 = _run(arrays, near, 1, grad)  # the plan has grown to the near view
    assert f3["layout_count"] > f3["num_rendered"]
    _assert_same(f3, fe, g3, ge, "after the plan grew")


def test_colour_only_backward_matches_zero_depth_and_alpha_planes():
    """Absent depth / alpha upstream gradients select the per-pixel backward
    that leaves their terms out; its gradients equal the general kernel's
    with zero planes (up to float atomic order)."""
    arrays = _scene(12003, 24)
    cam = camera.orbit_camera(45.0, 20.0, 2.5, 256, 256)
    grad = _grad(256, 256, 4)
    f = gh.forward(arrays, cam)
    t = f["_tensors"]
    means3D, opac, scales, rots, shs = arrays
    empty = torch.empty(0, device="cuda")
    zero = torch.zeros(1, 256, 256, device="cuda")
    bg = gh.dev(np.ones(3, np.float32))

    def bwd(dd, da):
        g = _C.rasterize_gaussians_backward(
            bg, gh.dev(means3D), t["radii"], empty, gh.dev(scales), gh.dev(rots), 1.0, empty, gh.dev(cam.viewmatrix),
            gh.dev(cam.projmatrix), float(cam.tanfovx), float(cam.tanfovy), gh.dev(grad), dd, da, gh.dev(shs), 3,
            gh.dev(cam.campos), t["geom"], f["num_rendered"], t["binb"], t["img"], t["alpha"], False, 0)
        return [x.cpu().numpy() for x in g]

    general = bwd(zero, zero)
    colour_only = bwd(empty, empty)
    for name, a, b in zip(parity.GRAD_NAMES, colour_only, general):
        chk = parity.grad_check(a, b, row_rtol=parity.SAME_IMPL_ROW_RTOL)
        assert chk["norm_rel"] <= 1e-6 and chk["n_bad"] == 0, (name, chk)
