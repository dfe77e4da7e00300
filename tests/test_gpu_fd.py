"""Central finite differences (h = 1e-3 relative) of the fp64 oracle forward
against the CUDA path's exact-mode gradients (grad_mode=1) on 256 seeded
parameters of a 600-Gaussian scene at 64x64.

A parameter whose +-h perturbation changes any blend decision (the oracle's
per-pixel decision signature) or the sorted instance list is skipped: the
rendered loss is piecewise smooth and the difference quotient straddles a
jump there.  The gradient of the CUDA path must agree with the difference
quotient to 2% of max(|fd|, 1e-3 * the largest gradient of that tensor)."""
import numpy as np
import pytest

import oracle
from word2world_b200 import camera, scenes

pytestmark = pytest.mark.gpu


def test_cuda_exact_gradients_match_central_differences():
    from tests.gpu_helpers import backward, forward
    sc = scenes.make_scene(600, seed=21)
    m, o, s, q, sh = sc.activate()
    S = 64
    cam = camera.orbit_camera(35.0, 20.0, 2.5, S, S)
    st = oracle.RasterSettings.from_camera(cam)
    rng = np.random.default_rng(256)
    g = rng.normal(size=(3, S, S)).astype(np.float32)
    arrays = (m, o, s, q, sh)
    fwd = forward(arrays, cam)
    b = backward(fwd, arrays, cam, g, grad_mode=1)
    an_all = dict(means3D=b["dL_dmeans3D"], scales=b["dL_dscales"], rotations=b["dL_drotations"],
                  opacities=b["dL_dopacity"], shs=b["dL_dsh"])
    base = dict(means3D=m, scales=s, rotations=q, opacities=o, shs=sh)
    gmax = {k: float(np.abs(v).max()) for k, v in an_all.items()}
    vis = np.nonzero(fwd["radii"] > 0)[0]
    names = list(base)
    checked, skipped, worst = 0, 0, 0.0
    for k in range(256):
        name = names[k % len(names)]
        arr = base[name]
        i = int(rng.choice(vis))
        idx = (i,) + tuple(int(rng.integers(0, d)) for d in arr.shape[1:])
        h = 1e-3 * max(abs(float(arr[idx])), 1e-2)
        ap, am = arr.copy(), arr.copy()
        ap[idx] += h
        am[idx] -= h
        hh = (float(ap[idx]) - float(am[idx])) / 2
        fp = oracle.forward(st, **{**base, name: ap}, precision="f64")
        fm = oracle.forward(st, **{**base, name: am}, precision="f64")
        if not (np.array_equal(fp["blend_signature"], fm["blend_signature"]) and
                np.array_equal(fp["point_list"], fm["point_list"])):
            skipped += 1
            continue
        fd = (oracle.scalar_loss(fp, g) - oracle.scalar_loss(fm, g)) / (2 * hh)
        an = float(np.asarray(an_all[name]).reshape(arr.shape)[idx])
        err = abs(fd - an) / max(abs(fd), 1e-3 * gmax[name], 1e-12)
        worst = max(worst, err)
        assert err <= 2e-2, (name, idx, fd, an)
        checked += 1
    print(f"finite differences: {checked} checked, {skipped} skipped, worst relative error {worst:.2e}")
    assert checked >= 128, (checked, skipped)
