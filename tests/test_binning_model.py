"""The premise of the binning path, checked on the oracle's own key emission
(no GPU): walking each Gaussian's owned slots with the Gaussians in stable
depth-bit order and placing the entries stably by tile gives exactly the
reference's sorted list (a stable sort of the emitted 64-bit keys).

Two facts carry it, both checked here on inputs with heavy spill
(compat_spill, large Gaussians): every Gaussian owns one contiguous run of
slots, and the runs appear in Gaussian order; so equal (tile, depth) keys
keep Gaussian order in the sort, and a Gaussian's own entries have distinct
tiles.
"""
import numpy as np
import pytest

import oracle
from word2world_b200 import camera, scenes


def _binning_model(f):
    uk, uv = f["unsorted_keys"], f["unsorted_vals"].astype(np.int64)
    R = len(uk)
    slots = np.arange(R)
    # one run of slots per Gaussian, runs in Gaussian order
    first = np.full(f["P"], -1, np.int64)
    last = np.full(f["P"], -1, np.int64)
    order_slots = np.argsort(uv, kind="stable")
    g_sorted = uv[order_slots]
    starts = np.r_[0, np.nonzero(np.diff(g_sorted))[0] + 1]
    ends = np.r_[starts[1:], R]
    for a, b in zip(starts, ends):
        run = order_slots[a:b]
        assert np.all(np.diff(run) == 1), "a Gaussian's slots are not contiguous"
        first[g_sorted[a]], last[g_sorted[a]] = run[0], run[-1]
    owners = g_sorted[starts]
    assert np.all(np.diff(first[owners]) > 0), "runs are not in Gaussian order"
    # each Gaussian's entries have distinct tiles
    tiles = (uk >> np.uint64(32)).astype(np.int64)
    pair = tiles * f["P"] + uv
    assert len(np.unique(pair)) == R
    # Gaussians by depth bits (stable), owned runs in that order, then a stable placement by tile
    dbits = (uk & np.uint64(0xffffffff)).astype(np.int64)
    gdepth = np.zeros(f["P"], np.int64)
    gdepth[uv] = dbits
    by_depth = np.argsort(gdepth[owners], kind="stable")
    seq = np.concatenate([np.arange(first[g], last[g] + 1) for g in owners[by_depth]]) if R else np.zeros(0, np.int64)
    placed = seq[np.argsort(tiles[seq], kind="stable")]
    return uk[placed], uv[placed].astype(np.uint32)


@pytest.mark.parametrize("case", [dict(P=3000, size=160, log_scale=(-4.0, -2.0), seed=3),
                                  dict(P=20000, size=256, log_scale=(-5.0, -3.0), seed=0),
                                  dict(P=1500, size=96, log_scale=(-3.0, -1.5), seed=7)])
def test_depth_ordered_placement_equals_the_sorted_keys(case):
    sc = scenes.make_scene(case["P"], seed=case["seed"], log_scale=case["log_scale"])
    m, o, s, q, sh = sc.activate()
    cam = camera.orbit_camera(30.0, 10.0, 2.5, case["size"], case["size"])
    f = oracle.forward(oracle.RasterSettings.from_camera(cam, compat_spill=True), m, s, q, o, sh)
    assert f["num_rendered"] > 0
    spilled = int(np.sum(f["candidates"] > 1))
    keys, vals = _binning_model(f)
    assert np.array_equal(keys, f["keys"])
    assert np.array_equal(vals, f["point_list"])
    print(f"R={f['num_rendered']} multi-writer slots {spilled}")
