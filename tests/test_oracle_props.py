"""Properties of the CPU oracle itself (no GPU)."""
import ctypes

import numpy as np
import pytest

import oracle
from word2world_b200 import camera, scenes


def _sorted(keys):
    k = keys.copy()
    v = np.arange(len(k), dtype=np.uint32)
    oracle.lib().orc_sort_pairs_u64(oracle._p(k), oracle._p(v), ctypes.c_longlong(len(k)))
    return k, v


@pytest.mark.parametrize("n", [0, 1, 2, 1000, 65537])
def test_sort_is_stable_sort(n):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 64, size=n, dtype=np.uint64) << np.uint64(rng.integers(0, 60))
    k, v = _sorted(keys)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order]) and np.array_equal(v, order.astype(np.uint32))


def test_scan():
    x = scenes.scan_workload(10000, seed=3)
    out = np.zeros_like(x)
    oracle.lib().orc_inclusive_scan_u32(oracle._p(x), oracle._p(out), ctypes.c_longlong(len(x)))
    assert np.array_equal(out, np.cumsum(x, dtype=np.uint64).astype(np.uint32))


@pytest.fixture(scope="module")
def fwd16k():
    sc = scenes.scene_16k(0)
    cam = camera.orbit_views(4, 2.5, 256, 256)[0]
    st = oracle.RasterSettings.from_camera(cam)
    m, o, s, q, sh = sc.activate()
    return oracle.forward(st, m, s, q, o, sh), (m, o, s, q, sh), st


def test_spill_model_invariants(fwd16k):
    f, arrays, st = fwd16k
    R = f["num_rendered"]
    assert R == int(f["tiles"].sum())
    # every slot has at least one candidate writer (emission covers allocation)
    assert np.all(f["candidates"] >= 1)
    # about a quarter of Gaussians emit beyond their allocation
    assert 0.0 < (f["candidates"] > 1).mean() < 0.5
    # the clean mode emits exactly the allocation: one writer per slot
    st2 = oracle.RasterSettings(**{**st.__dict__, "compat_spill": False})
    m, o, s, q, sh = arrays
    f2 = oracle.forward(st2, m, s, q, o, sh)
    assert np.all(f2["candidates"] == 1)
    assert f2["num_rendered"] == R


def test_keys_sorted_and_ranges_consistent(fwd16k):
    f, _, st = fwd16k
    k = f["keys"]
    assert np.all(k[1:] >= k[:-1])
    tiles = (k >> np.uint64(32)).astype(np.int64)
    for t in np.unique(tiles)[:50]:
        s, e = f["ranges"][t]
        assert np.all(tiles[s:e] == t) and e - s == np.sum(tiles == t)


def test_fp32_vs_fp64(fwd16k):
    """The fp64 re-evaluation redoes the arithmetic on the fp32 path's sorted
    lists: re-sorting in fp64 legitimately swaps Gaussians whose fp32 depths
    tie or nearly tie (NDC depths ~0.996 are 6e-8 apart in fp32), and blend
    order changes colour."""
    import parity
    f, arrays, st = fwd16k
    m, o, s, q, sh = arrays
    g64 = oracle.preprocess(st, m, s, q, o, sh, precision="f64")
    d = oracle.blend(st, g64, f["ranges"], f["point_list"], precision="f64")
    assert np.array_equal(f["n_contrib"], d["n_contrib"])
    for k in ("color", "alpha", "depth_img"):
        e = parity.err_stats(f[k], d[k])
        assert e["n_bad"] == 0, (k, e)


def test_finite_differences_exact_mode():
    """Central differences of the fp64 forward vs the exact-mode gradient, on
    parameters whose +-h perturbation leaves every blend decision unchanged."""
    sc = scenes.make_scene(300, seed=8)
    m, o, s, q, sh = sc.activate()
    cam = camera.orbit_camera(60.0, 15.0, 2.5, 48, 48)
    st = oracle.RasterSettings.from_camera(cam)
    rng = np.random.default_rng(0)
    g = rng.normal(size=(3, 48, 48)).astype(np.float32)
    f = oracle.forward(st, m, s, q, o, sh, precision="f64")
    b = oracle.backward(f, g, mode="exact")
    base = dict(means3D=m, scales=s, rotations=q, opacities=o, shs=sh)
    key = dict(means3D="dL_dmeans3D", scales="dL_dscales", rotations="dL_drotations", opacities="dL_dopacity",
               shs="dL_dsh")
    vis = np.nonzero(f["radii"] > 0)[0]
    checked = 0
    for name, arr in base.items():
        for _ in range(6):
            i = int(rng.choice(vis))
            idx = (i,) + tuple(int(rng.integers(0, d)) for d in arr.shape[1:])
            h = 1e-4 * max(abs(float(arr[idx])), 1e-2)
            ap, am = arr.copy(), arr.copy()
            ap[idx] += h
            am[idx] -= h
            hh = (float(ap[idx]) - float(am[idx])) / 2
            fp = oracle.forward(st, **{**dict(means3D=m, scales=s, rotations=q, opacities=o, shs=sh), name: ap},
                                precision="f64")
            fm = oracle.forward(st, **{**dict(means3D=m, scales=s, rotations=q, opacities=o, shs=sh), name: am},
                                precision="f64")
            if not (np.array_equal(fp["blend_signature"], fm["blend_signature"]) and
                    np.array_equal(fp["point_list"], fm["point_list"])):
                continue
            fd = (oracle.scalar_loss(fp, g) - oracle.scalar_loss(fm, g)) / (2 * hh)
            an = float(np.asarray(b[key[name]]).reshape(arr.shape)[idx]) if name != "opacities" else \
                float(b["dL_dopacity"][i, 0])
            assert abs(fd - an) <= 1e-3 * max(1.0, abs(fd)), (name, idx, fd, an)
            checked += 1
    assert checked >= 15


@pytest.mark.parametrize("case", ["empty", "culled", "one"])
def test_empty_culled_and_single_inputs(case):
    """The oracle on the edge inputs the GPU tests hand it: no Gaussians, every
    Gaussian at the camera centre (culled by the near test), one Gaussian.
    Nothing rendered leaves the background, zero contributor counts,
    transmittance one and zero gradients; one Gaussian gives a sorted list of
    its own tiles."""
    P = {"empty": 0, "culled": 500, "one": 1}[case]
    sc = scenes.make_scene(P, seed=9)
    m, o, s, q, sh = sc.activate()
    cam = camera.orbit_camera(30.0, 10.0, 2.5, 64, 48)
    if case == "culled":
        m = np.repeat(-np.asarray(cam.campos, np.float32)[None], P, axis=0)
    st = oracle.RasterSettings.from_camera(cam, bg=(0.25, 0.5, 1.0))
    f = oracle.forward(st, m, s, q, o, sh)
    g = np.random.default_rng(4).normal(size=(3, 48, 64)).astype(np.float32)
    b = oracle.backward(f, g)
    if case != "one":
        assert f["num_rendered"] == 0 and np.all(np.asarray(f["radii"]) == 0)
        assert np.array_equal(np.asarray(f["color"]), np.broadcast_to(np.float32([0.25, 0.5, 1.0])[:, None, None],
                                                                        (3, 48, 64)))
        assert np.all(np.asarray(f["n_contrib"]) == 0) and np.all(np.asarray(f["alpha"]) == 0)
        for k, v in b.items():
            if k.startswith(("dL_", "abs_")):  # every gradient and its sum of |terms|
                assert not np.any(np.asarray(v)), k
        return
    R = f["num_rendered"]
    assert R == int(np.asarray(f["tiles"])[0]) > 0
    keys = np.asarray(f["keys"])[:R]
    assert np.all(np.diff(keys.astype(np.int64)) > 0)  # one Gaussian: distinct tiles, ascending
    assert np.all(np.asarray(f["point_list"])[:R] == 0)
