"""Batched calls (many views of many scenes, one launch per stage) against
the single-view entry points on the same inputs: images, radii and
contributor counts bit-identical per item, gradients equal up to float
atomic order."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

import parity  # noqa: E402
from word2world_b200 import _C, camera, scenes  # noqa: E402
from word2world_b200.batch import BatchRenderer, Scene, View  # noqa: E402

DEV = "cuda"


def _setup():
    specs = [dict(P=2048, seed=3, layout="shell"), dict(P=8192, seed=4, layout="ball"),
             dict(P=6000, seed=5, layout="shell", log_scale=(-4.0, -2.5))]
    scs = [Scene.from_arrays(scenes.make_scene(**sp).activate(), DEV) for sp in specs]
    views = [View(0, camera.orbit_camera(0.0, 0.0, 2.5, 128, 128)),
             View(1, camera.orbit_camera(40.0, 10.0, 2.5, 160, 96), (0.2, 0.5, 1.0)),
             View(0, camera.orbit_camera(200.0, -20.0, 2.5, 128, 128)),
             View(2, camera.orbit_camera(90.0, 30.0, 2.5, 256, 256)),
             View(1, camera.orbit_camera(300.0, 0.0, 2.5, 64, 200))]
    return scs, views


def _plain(sc, view):
    c = view.camera
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(DEV)
    bg = torch.tensor(view.background, dtype=torch.float32, device=DEV)
    return _C.rasterize_gaussians(sc.shs, c.focal_y, sc.scales, sc.means3D, t(c.projmatrix), sc.sh_degree,
                                  sc.opacities, sc.rotations, t(c.campos), t(c.viewmatrix), c.focal_x, c.height,
                                  c.width, bg, True), bg


@pytest.mark.parametrize("grad_mode,reuse,queue", [("reference", False, 0), ("exact", False, 0), ("reference", True, 0),
                                                   ("reference", False, 1)])
def test_batch_matches_single_views(grad_mode, reuse, queue):
    """queue = 1: the batched blend is the persistent one, its queue holding
    every item's tiles."""
    from word2world_b200 import autotune
    prev = autotune.apply({"blend_queue": queue})
    try:
        _batch_matches_single_views(grad_mode, reuse)
    finally:
        autotune.apply(prev)


def _batch_matches_single_views(grad_mode, reuse):
    scs, views = _setup()
    br = BatchRenderer(grad_mode=grad_mode, reuse_buffers=reuse)
    rng = np.random.default_rng(11)
    grads = [torch.from_numpy(rng.normal(size=(3, v.camera.height, v.camera.width)).astype(np.float32)).to(DEV)
             for v in views]
    if reuse:  # leave another batch's contents in the workspace first
        warm = br.forward(scs, views[::-1])
        br.backward(warm, [torch.randn_like(g) for g in grads[::-1]])
    res = br.forward(scs, views)
    g = br.backward(res, grads, per_element=True)
    torch.cuda.synchronize()
    npix_before = 0
    img_nc = res.state["img"][:4 * res.state["npix"]].view(torch.int32)
    for v, view in enumerate(views):
        sc = scs[view.scene]
        (R, color, depth, alpha, radii, geom, binb, img), bg = _plain(sc, view)
        c = view.camera
        for name, a, b in (("color", res.color[v], color), ("depth", res.depth[v], depth), ("alpha", res.alpha[v], alpha),
                           ("radii", res.radii[v], radii)):
            assert parity.bit_mismatch(a.cpu().numpy(), b.cpu().numpy()) == 0, (v, name)
        hw = c.width * c.height
        nc_b = img_nc[npix_before:npix_before + hw].cpu().numpy()
        nc_p = img[:4 * hw].view(torch.int32).cpu().numpy()
        assert parity.bit_mismatch(nc_b, nc_p) == 0, (v, "n_contrib")
        npix_before += hw
        # the single-view backward on the same inputs
        empty = torch.empty(0, device=DEV)
        zero = torch.zeros(1, c.height, c.width, device=DEV)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(DEV)
        gp = _C.rasterize_gaussians_backward(
            bg, sc.means3D, radii, empty, sc.scales, sc.rotations, 1.0, empty, t(c.viewmatrix), t(c.projmatrix),
            c.tanfovx, c.tanfovy, grads[v], zero, zero, sc.shs, sc.sh_degree, t(c.campos), geom, R, binb, img, alpha,
            False, 0 if grad_mode == "reference" else 1)
        for name, a, b in zip(parity.GRAD_NAMES, g["per_item"][v], gp):
            chk = parity.grad_check(a.cpu().numpy(), b.cpu().numpy(), row_rtol=parity.SAME_IMPL_ROW_RTOL)
            assert chk["norm_rel"] <= 1e-5, (v, name, chk)
            assert chk["n_bad"] == 0, (v, name, chk)


def test_batch_scene_gradient_is_sum_over_its_views():
    scs, views = _setup()
    br = BatchRenderer()
    res = br.forward(scs, views)
    grads = [torch.ones(3, v.camera.height, v.camera.width, device=DEV) for v in views]
    g = br.backward(res, grads, per_element=True)
    for s in range(len(scs)):
        items = [v for v, view in enumerate(views) if view.scene == s]
        want = sum(g["per_item"][v][3] for v in items)
        got = g["means3D"][g["groups"].index(s)]
        assert torch.allclose(got, want, rtol=1e-6, atol=1e-7)


def _views_with_straddling_groups():
    """The _setup views reordered so that the first group (scene 2, 6000
    Gaussians) ends inside a warp of the grouped pass: rows 5984-6015 mix
    scene 2 and scene 0."""
    scs, views = _setup()
    return scs, [views[3], views[0], views[1], views[2], views[4]]


@pytest.mark.parametrize("grad_mode", ["reference", "exact"])
def test_grouped_pass_equals_group_sum(grad_mode):
    """The grouped per-Gaussian pass, run over the per-element accumulators a
    per-element backward left, against w2w_group_sum's sums of that
    backward's per-element gradients: the same inputs and summation order; the
    per-view arithmetic, inlined into another kernel, may fuse a multiply-add
    differently, so values agree to a few ulps (no atomic order is involved)."""
    import ctypes
    from word2world_b200.batch import lib
    scs, views = _views_with_straddling_groups()
    br = BatchRenderer(grad_mode=grad_mode)
    res = br.forward(scs, views)
    rng = np.random.default_rng(5)
    grads = [torch.from_numpy(rng.normal(size=(3, v.camera.height, v.camera.width)).astype(np.float32)).to(DEV)
             for v in views]
    g = br.backward(res, grads, per_element=True)
    lb, st = br._last_backward, res.state
    total, M = lb["total"], st["M"]
    outs = {name: torch.full((total, *shp), float("nan"), device=DEV)
            for name, shp in (("means3D", (3,)), ("opacities", (1,)), ("scales", (3,)), ("rotations", (4,)),
                              ("shs", (M, 3)))}
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib().w2w_batch_gaussians_grouped(
        st["arr"], st["n"], p(st["geom"]), p(st["radii"]), br.grad_mode, p(lb["scratch"]),
        ctypes.c_size_t(lb["scratch"].numel()), p(lb["g_m2"]), p(lb["g_col"]), p(lb["g_op"]), p(lb["tables"]),
        lb["G"], ctypes.c_longlong(total), p(outs["means3D"]), p(outs["opacities"]), p(outs["scales"]),
        p(outs["rotations"]), p(outs["shs"]), stream)
    assert rc == 0
    torch.cuda.synchronize()
    assert g["groups"] == [2, 0, 1]
    for name in outs:
        want = torch.cat([x.reshape(x.shape[0], -1) for x in g[name]]).cpu().numpy()
        got = outs[name].reshape(total, -1).cpu().numpy()
        chk = parity.grad_check(got, want, row_rtol=parity.SAME_IMPL_ROW_RTOL)
        assert chk["norm_rel"] <= 1e-6 and chk["n_bad"] == 0, (name, chk)


@pytest.mark.parametrize("grad_mode", ["reference", "exact"])
def test_grouped_backward_sums_the_views(grad_mode):
    """The default batched backward (grouped pass) against the per-item
    gradients of a per-element backward summed per scene: equal up to the
    float atomic order of the per-pixel pass."""
    scs, views = _views_with_straddling_groups()
    br = BatchRenderer(grad_mode=grad_mode)
    res = br.forward(scs, views)
    rng = np.random.default_rng(6)
    grads = [torch.from_numpy(rng.normal(size=(3, v.camera.height, v.camera.width)).astype(np.float32)).to(DEV)
             for v in views]
    ref = br.backward(res, grads, per_element=True)
    got = br.backward(res, grads)
    assert got["groups"] == ref["groups"]
    for k, s in enumerate(got["groups"]):
        items = [v for v, view in enumerate(views) if view.scene == s]
        for name, col in (("means3D", 3), ("scales", 6), ("rotations", 7), ("shs", 5), ("opacities", 2)):
            want = sum(ref["per_item"][v][col].double() for v in items).float()
            chk = parity.grad_check(got[name][k].reshape(want.shape).cpu().numpy(), want.cpu().numpy(),
                                    row_rtol=parity.SAME_IMPL_ROW_RTOL)
            assert chk["norm_rel"] <= 1e-5, (s, name, chk)
