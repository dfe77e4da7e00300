"""The drop-in Python boundary: ``_render_gaussians_inline`` (the
torch.autograd.Function of Renderer.py:28-110) and ``Renderer.render``
(Renderer.py:119-192) against the binding they wrap.

* the autograd Function's image, radii, depth and alpha are the binding's
  forward outputs bit for bit, and the gradients autograd delivers to its
  inputs are the binding's backward outputs for the same upstream gradient;
* ``Renderer.render`` is the reference's activation preamble (sigmoid
  opacity, exp scales, normalised quaternion, concatenated SH) followed by
  that Function: its image equals the Function's on torch-activated
  parameters bit for bit, and the raw parameters' gradients equal autograd
  through the same torch preamble;
* the image agrees with the oracle on the same activated parameters."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

import oracle  # noqa: E402
import parity  # noqa: E402
from word2world_b200 import _C, camera, scenes  # noqa: E402
from word2world_b200.renderer import GaussianParams, Renderer, _render_gaussians_inline  # noqa: E402

DEV = "cuda"


def _setup(P=6000, S=128, seed=3):
    sc = scenes.make_scene(P, seed=seed, layout="ball")
    cam = camera.orbit_camera(40.0, 10.0, 2.5, S, S)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(DEV)
    return sc, cam, t


@pytest.mark.parametrize("grad_mode", ["reference", "exact"])
def test_autograd_function_matches_binding(grad_mode):
    sc, cam, t = _setup()
    m, o, s, q, sh = sc.activate()
    S = cam.width
    leaves = [t(x).requires_grad_(True) for x in (m, sh, o, s, q)]
    means3D, shs, opac, scales, rots = leaves
    means2D = torch.zeros_like(means3D, requires_grad=True)
    bg = torch.ones(3, device=DEV)
    V, Pm, C = t(cam.viewmatrix), t(cam.projmatrix), t(cam.campos)
    color, radii, depth, alpha = _render_gaussians_inline(
        means3D, means2D, shs, None, opac, scales, rots, None, bg, 1.0, V, Pm, cam.tanfovx, cam.tanfovy, 3, C,
        image_height=S, image_width=S, grad_mode=grad_mode)
    R, color_b, depth_b, alpha_b, radii_b, geom, binb, img = _C.rasterize_gaussians(
        shs.detach(), cam.focal_y, scales.detach(), means3D.detach(), Pm, 3, opac.detach(), rots.detach(), C, V,
        cam.focal_x, S, S, bg, True)
    for a, b in ((color, color_b), (depth, depth_b), (alpha, alpha_b), (radii, radii_b)):
        assert parity.bit_mismatch(a.detach().cpu().numpy(), b.cpu().numpy()) == 0
    g = torch.randn(3, S, S, device=DEV, generator=torch.Generator(device=DEV).manual_seed(1))
    torch.autograd.backward([color], [g])
    z = torch.zeros(1, S, S, device=DEV)
    empty = torch.empty(0, device=DEV)
    gb = _C.rasterize_gaussians_backward(bg, means3D.detach(), radii_b, empty, scales.detach(), rots.detach(), 1.0,
                                         empty, V, Pm, cam.tanfovx, cam.tanfovy, g, z, z, shs.detach(), 3, C, geom,
                                         R, binb, img, alpha_b, False, 0 if grad_mode == "reference" else 1)
    want = dict(means2D=gb[0], opac=gb[2], means3D=gb[3], shs=gb[5], scales=gb[6], rots=gb[7])
    got = dict(means2D=means2D.grad, opac=opac.grad, means3D=means3D.grad, shs=shs.grad, scales=scales.grad,
               rots=rots.grad)
    for k in want:
        chk = parity.grad_check(got[k].cpu().numpy(), want[k].cpu().numpy(), row_rtol=parity.SAME_IMPL_ROW_RTOL)
        assert chk["norm_rel"] <= 1e-5 and chk["n_bad"] == 0, (k, chk)


@pytest.mark.parametrize("grad_mode,degree", [("reference", 3), ("exact", 3), ("reference", 0)])
def test_renderer_render_is_preamble_plus_function(grad_mode, degree):
    """In "reference" mode ``Renderer.render`` runs the raw-parameter Function
    (preamble folded into the projection and the per-Gaussian backward); in
    "exact" mode the fused activation kernels and the plain Function."""
    sc, cam, t = _setup(seed=4)
    S = cam.width
    params = GaussianParams.from_scene(sc, device=DEV)
    with torch.no_grad():  # a few degenerate quaternions: the normalisation's 1e-12 floor
        params.quaternion[:7] = 0.0
        params.quaternion[7:14] *= 1e-20
    r = Renderer(params, sh_degree=degree, grad_mode=grad_mode)
    out = r.render(cam.fovx, cam.fovy, t(cam.viewmatrix), t(cam.projmatrix), t(cam.campos), S, S)
    assert set(out) >= {"image", "accum_grads", "avaialble_pts", "available_pts"}
    g = torch.randn(3, S, S, device=DEV, generator=torch.Generator(device=DEV).manual_seed(2))
    (out["image"] * g).sum().backward()
    got = [p.grad.clone() for p in params.parameters()]

    # the same preamble written out with torch ops, then the Function
    raw = [p.detach().clone().requires_grad_(True) for p in params.parameters()]
    mean, sh_dc, sh_ac, opac_l, svec, quat = raw
    shs = torch.cat((sh_dc, sh_ac), dim=1)
    means2D = torch.zeros_like(mean, requires_grad=True)
    image, radii, _, _ = _render_gaussians_inline(
        mean, means2D, shs, None, torch.sigmoid(opac_l), torch.exp(svec), torch.nn.functional.normalize(quat), None,
        torch.ones(3, device=DEV), 1, t(cam.viewmatrix), t(cam.projmatrix), np.tan(cam.fovx / 2),
        np.tan(cam.fovy / 2), degree, t(cam.campos), image_height=S, image_width=S, grad_mode=grad_mode)
    assert parity.bit_mismatch(out["image"].detach().cpu().numpy(), image.detach().cpu().numpy()) == 0
    assert torch.equal(out["available_pts"], radii > 0)
    (image * g).sum().backward()
    for name, a, b in zip(("mean", "sh_dc", "sh_ac", "opacity", "svec", "quaternion"), got, raw):
        a, b = a.cpu().numpy(), b.grad.cpu().numpy()
        if name == "quaternion":  # at the floor torch's clamp has a kink; both sides take g / 1e-12
            # g is summed by atomics in either order: relative to its row's largest element
            row = np.abs(b[:14]).max(axis=1, keepdims=True)
            assert np.all(np.abs(a[:14] - b[:14]) <= 1e-5 * (np.abs(b[:14]) + row)), (a[:14], b[:14])
        chk = parity.grad_check(a, b, row_rtol=parity.SAME_IMPL_ROW_RTOL)
        assert chk["norm_rel"] <= 1e-5 and chk["n_bad"] == 0, (name, chk)

    # and the image is the oracle's on the activated parameters
    n = lambda x: x.detach().cpu().numpy()
    m, o, s, q, sh = (n(mean), n(torch.sigmoid(opac_l)), n(torch.exp(svec)),
                      n(torch.nn.functional.normalize(quat)), n(shs))
    f = oracle.forward(oracle.RasterSettings.from_camera(cam, degree=degree), m, s, q, o, sh)
    np.testing.assert_allclose(out["image"].detach().cpu().numpy(), f["color"], rtol=1e-4, atol=1e-5)


def test_fused_activation_matches_torch():
    """The fused preamble is bit-identical to the torch operations forward and
    equal up to rounding backward, including zero and huge quaternions and
    saturating logits."""
    from word2world_b200.renderer import activate
    gen = torch.Generator(device=DEV).manual_seed(5)
    P = 200_003
    logit = (torch.randn(P, 1, device=DEV, generator=gen) * 6).requires_grad_(True)
    svec = (torch.randn(P, 3, device=DEV, generator=gen) * 3).requires_grad_(True)
    q = torch.randn(P, 4, device=DEV, generator=gen)
    q[:1000] = 0.0
    q[1000:2000] *= 1e-20
    q[2000:3000] *= 1e15
    q.requires_grad_(True)
    dc = torch.randn(P, 1, 3, device=DEV, generator=gen).requires_grad_(True)
    ac = torch.randn(P, 15, 3, device=DEV, generator=gen).requires_grad_(True)
    got = activate(logit, svec, q, dc, ac)
    want = (torch.sigmoid(logit), torch.exp(svec), torch.nn.functional.normalize(q), torch.cat((dc, ac), dim=1))
    for a, b in zip(got, want):
        assert a.shape == b.shape
        assert parity.bit_mismatch(a.detach().cpu().numpy(), b.detach().cpu().numpy()) == 0
    gs = [torch.randn(t.shape, device=DEV, generator=gen) for t in want]
    gg = torch.autograd.grad(got, (logit, svec, q, dc, ac), gs)
    gw = torch.autograd.grad(want, (logit, svec, q, dc, ac), gs)
    for name, a, b in zip(("logit", "svec", "quaternion", "sh_dc", "sh_ac"), gg, gw):
        a, b = a.cpu().numpy().reshape(P, -1), b.cpu().numpy().reshape(P, -1)
        if name == "quaternion":  # away from the 1e-12 floor, where torch's clamp has a kink
            a, b = a[1000:], b[1000:]
        chk = parity.grad_check(a, b, row_rtol=parity.SAME_IMPL_ROW_RTOL)
        assert chk["norm_rel"] <= 1e-6 and chk["n_bad"] == 0, (name, chk)


def test_densification_stats_match_masked_torch():
    """Two renders' statistics accumulate as the reference's masked torch
    updates do (gaussians_handler.py:116-118)."""
    from word2world_b200.renderer import DensificationStats
    gen = torch.Generator(device=DEV).manual_seed(6)
    P = 100_001
    st = DensificationStats(P)
    acc_ref = torch.zeros(P, 1, device=DEV)
    cnt_ref = torch.zeros(P, 1, device=DEV)
    for _ in range(2):
        g = torch.randn(P, 3, device=DEV, generator=gen)
        radii = torch.randint(0, 3, (P,), device=DEV, generator=gen, dtype=torch.int32)
        st.collect(g, radii)
        f = radii > 0
        cnt_ref[f] += 1
        acc_ref[f] += torch.norm(g[f, :2], dim=-1, keepdim=True)
    assert torch.equal(st.counter, cnt_ref)
    torch.testing.assert_close(st.mean_gradient_accum, acc_ref, rtol=1e-6, atol=0)


def test_ply_round_trip_renders_identically(tmp_path):
    """Parameters saved in the reference's PLY layout and loaded back, as
    GaussianParams or as a resident serving scene, render the same image."""
    import os
    from word2world_b200.batch import BatchRenderer, Scene, View
    sc, cam, t = _setup(P=3000, seed=8)
    S = cam.width
    params = GaussianParams.from_scene(sc, device=DEV)
    path = os.path.join(tmp_path, "scene.ply")
    params.save_ply(path)
    again = GaussianParams.load_ply(path, device=DEV)
    for a, b in zip(params.parameters(), again.parameters()):
        assert torch.equal(a.detach(), b.detach())
    args = (cam.fovx, cam.fovy, t(cam.viewmatrix), t(cam.projmatrix), t(cam.campos), S, S)
    img0 = Renderer(params, sh_degree=3).render(*args)["image"].detach()
    img1 = Renderer(again, sh_degree=3).render(*args)["image"].detach()
    assert torch.equal(img0, img1)
    res = BatchRenderer().forward([Scene.from_ply(path, device=DEV)], [View(0, cam)])
    assert parity.bit_mismatch(res.color[0].cpu().numpy(), img0.cpu().numpy()) == 0


def test_views_on_separate_streams_match_one_stream():
    """The binding launches on the current stream and waits only on it, so the
    views of a step may run on separate streams: the images are the
    single-stream images bit for bit and the accumulated leaf gradients agree
    up to the order of the atomic additions."""
    sc, cam0, t = _setup(seed=6)
    from word2world_b200 import camera
    cams = camera.orbit_views(3, 2.5, cam0.width, cam0.height)
    m, o, s, q, sh = sc.activate()
    leaves = [t(x).requires_grad_(True) for x in (m, sh, o, s, q)]
    means3D, shs, opac, scales, rots = leaves
    means2D = torch.zeros_like(means3D, requires_grad=True)
    bg = torch.ones(3, device=DEV)
    S = cam0.width
    gen = torch.Generator(device=DEV).manual_seed(7)
    gs = [torch.randn(3, S, S, device=DEV, generator=gen) for _ in cams]
    ct = [(t(c.viewmatrix), t(c.projmatrix), t(c.campos), c.tanfovx, c.tanfovy) for c in cams]

    def view(v):
        V, Pm, C, tx, ty = ct[v]
        color, _, _, _ = _render_gaussians_inline(means3D, means2D, shs, None, opac, scales, rots, None, bg, 1.0, V,
                                                  Pm, tx, ty, 3, C, image_height=S, image_width=S)
        torch.autograd.backward([color], [gs[v]])
        return color.detach()

    def run(streams):
        for x in leaves + [means2D]:
            x.grad = None
        main = torch.cuda.current_stream()
        imgs = []
        for v in range(len(cams)):
            if streams is None:
                imgs.append(view(v))
                continue
            streams[v].wait_stream(main)
            with torch.cuda.stream(streams[v]):
                imgs.append(view(v))
        if streams is not None:
            for st in streams:
                main.wait_stream(st)
        torch.cuda.synchronize()
        return [i.cpu().numpy() for i in imgs], [x.grad.cpu().numpy() for x in leaves + [means2D]]

    img1, g1 = run(None)
    img2, g2 = run([torch.cuda.Stream() for _ in cams])
    for a_, b_ in zip(img1, img2):
        assert parity.bit_mismatch(a_, b_) == 0
    for name, a_, b_ in zip(("means3D", "shs", "opacity", "scales", "rotations", "means2D"), g1, g2):
        chk = parity.grad_check(a_, b_, row_rtol=parity.SAME_IMPL_ROW_RTOL)
        assert chk["norm_rel"] <= 1e-5 and chk["n_bad"] == 0, (name, chk)


def test_densification_fused_into_the_backward_matches_collect():
    """Renderer(densification=stats): each render's backward accumulates the
    statistics in its per-Gaussian pass; over three views they equal collect
    calls on the same renders' gradients after each backward, exactly (the
    same arithmetic on the same values, in the same order on one stream)."""
    from word2world_b200 import camera
    from word2world_b200.renderer import DensificationStats
    sc, cam0, t = _setup(P=20000, S=256, seed=9)
    cams = camera.orbit_views(3, 2.5, 256, 256)
    gen = torch.Generator(device=DEV).manual_seed(8)
    gs = [torch.randn(3, 256, 256, device=DEV, generator=gen) for _ in cams]
    params = GaussianParams.from_scene(sc, device=DEV)
    fused = DensificationStats(params.mean.shape[0])
    collected = DensificationStats(params.mean.shape[0])
    r = Renderer(params, sh_degree=3, densification=fused)
    for c, g in zip(cams, gs):
        out = r.render(c.fovx, c.fovy, t(c.viewmatrix), t(c.projmatrix), t(c.campos), 256, 256)
        (out["image"] * g).sum().backward()
        collected.collect(out["accum_grads"], out["available_pts"].to(torch.int32))
    torch.cuda.synchronize()
    assert torch.count_nonzero(collected.counter) > 0
    assert torch.equal(fused.counter, collected.counter)
    assert torch.equal(fused.mean_gradient_accum, collected.mean_gradient_accum)
    with pytest.raises(ValueError):
        Renderer(GaussianParams.from_scene(sc, device=DEV), grad_mode="exact", densification=fused)
