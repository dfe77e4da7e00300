"""Autotuner: coordinate descent over the library's launch-shape knobs with a
fake timer (CPU), the knob setter's validation, and (GPU) identical results
under every knob setting."""
import json

import numpy as np
import pytest

torch = pytest.importorskip("torch")

try:
    from word2world_b200 import _C, autotune
except ImportError:  # the extension is not built here
    _C = None


@pytest.fixture
def restore():
    if _C is None:
        pytest.skip("extension not built")
    before = autotune.current()
    yield
    autotune.apply(before)


def test_knob_setter_validates(restore):
    knobs = autotune.current()
    assert set(knobs) == set(autotune.CANDIDATES)
    with pytest.raises(ValueError):
        _C.tune_set("blend_warps", 5)
    with pytest.raises(ValueError):
        _C.tune_set("no_such_knob", 1)
    with pytest.raises(ValueError):
        _C.tune_set("blend_stage", 2)  # 0: records gathered into registers, 1: copied by cp.async
    assert autotune.current() == knobs
    prev = autotune.apply({"backward_ways": 3})
    assert prev == {"backward_ways": knobs["backward_ways"]} and autotune.current()["backward_ways"] == 3


def test_descent_finds_the_cheapest_setting_and_caches_it(restore, tmp_path):
    # a cost model over the knobs: its minimum is blend_warps 8, backward_split 2, backward_ways 3, binning 1,
    # blend_queue 1
    def cost():
        k = autotune.current()
        return (1.0 + (0.0 if k["blend_warps"] == 8 else 0.3) + abs(k["backward_split"] - 2) * 0.1 +
                (0.0 if k["backward_ways"] == 3 else 0.05) + (0.0 if k["binning"] == 1 else 0.02) +
                (0.0 if k["blend_queue"] == 1 else 0.04))

    path = str(tmp_path / "tune.json")
    t = autotune.Autotuner(path=path, timer=lambda step: cost())
    autotune.apply({"blend_warps": 4, "backward_split": 4, "backward_ways": 2, "binning": 0, "blend_queue": 0,
                    "preprocess_blocks": 4, "blend_stage": 1})
    best = t.tune("bucket", step=None)
    # preprocess_blocks and blend_stage do not enter the cost: they keep their starting values
    assert best == {"blend_warps": 8, "backward_split": 2, "backward_ways": 3, "binning": 1, "blend_queue": 1,
                    "preprocess_blocks": 4, "blend_stage": 1}
    assert autotune.current() == best
    saved = json.load(open(path))
    assert saved["bucket"]["blend_warps"] == 8
    # a second tuner reads the cache and applies it without timing anything
    autotune.apply({"blend_warps": 4, "backward_split": 4, "backward_ways": 2, "binning": 0, "blend_queue": 0,
                    "preprocess_blocks": 4, "blend_stage": 1})
    t2 = autotune.Autotuner(path=path, timer=lambda step: pytest.fail("timed a cached bucket"))
    assert t2.ensure("bucket", step=None) == best and autotune.current() == best


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")
def test_every_knob_setting_gives_the_same_results(restore):
    import gpu_helpers as gh
    import parity
    from word2world_b200 import camera, scenes
    arrays = scenes.make_scene(20000, seed=8, layout="ball").activate()
    cam = camera.orbit_camera(60.0, 15.0, 2.5, 256, 256)
    g = np.random.default_rng(3).normal(size=(3, 256, 256)).astype(np.float32)
    base = None
    for warps, split, ways, binning, queue, pre, stage in ((4, 4, 2, 0, 0, 4, 1), (8, 4, 2, 0, 0, 3, 1),
                                                           (4, 0, 2, 1, 0, 2, 0), (4, 8, 3, 1, 1, 4, 1),
                                                           (8, 8, 2, 1, 1, 2, 0), (4, 4, 3, 0, 1, 3, 0),
                                                           (8, 4, 2, 0, 1, 4, 1), (4, 2, 2, 0, 0, 4, 0),
                                                           (8, 2, 2, 0, 0, 4, 0)):
        autotune.apply({"blend_warps": warps, "backward_split": split, "backward_ways": ways, "binning": binning,
                        "blend_queue": queue, "preprocess_blocks": pre, "blend_stage": stage})
        f = gh.forward(arrays, cam)
        b = gh.backward(f, arrays, cam, g, grad_mode=0)
        if base is None:
            base = (f, b)
            continue
        for k in ("color", "alpha", "depth_img", "n_contrib", "keys", "point_list"):
            assert parity.bit_mismatch(f[k], base[0][k]) == 0, (warps, split, ways, binning, queue, k)
        for k in parity.GRAD_NAMES:
            c = parity.grad_check(b[k], base[1][k], row_rtol=parity.SAME_IMPL_ROW_RTOL)
            assert c["norm_rel"] <= 1e-5, (warps, split, ways, binning, k, c)
