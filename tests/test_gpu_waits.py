"""Failure path of the bounded device waits, on the GPU, without a fault.

The single-pass scans and the sort's passes wait for their predecessor tiles
with an iteration limit.  A test hook makes one tile's CTA skip publishing
its status (a flag nothing else sets), so the waits behind it run out at a
lowered limit.  Checked: the stand-alone scans and the sort report
W2W_ERR_TIMEOUT (through their error words, in checked mode through their
return value, and through the torch binding); a render's deferred error word
raises on the next check; the projection pass's fused scan makes the forward
raise at once.  Afterwards every path runs clean again with correct results.
Nothing traps, faults or hangs: every wait ends at its limit, and ids the
inconsistent sort output leaves in a point list are skipped, never read.
"""
import ctypes
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

import gpu_helpers as gh  # noqa: E402
from word2world_b200 import _C, camera, scenes  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "word2world_b200", "libw2w_raster.so")
W2W_ERR_TIMEOUT = 4
STAGE_SCAN, STAGE_SORT, STAGE_PREPROCESS = 0, 1, 2


def _lib():
    lib = ctypes.CDLL(LIB)
    vp, ll, sz = ctypes.c_void_p, ctypes.c_longlong, ctypes.c_size_t
    lib.w2w_scan_u32.argtypes = [vp, vp, ll, ctypes.c_int, vp, sz, vp]
    lib.w2w_scan_u32_noalloc.argtypes = [vp, vp, ll, ctypes.c_int, vp]
    lib.w2w_scan_scratch_bytes.argtypes = [ll]
    lib.w2w_scan_scratch_bytes.restype = sz
    lib.w2w_scratch_error.argtypes = [vp, vp]
    lib.w2w_scan_noalloc_error.argtypes = [vp]
    lib.w2w_set_error_check.argtypes = [ctypes.c_int]
    return lib


class hooked:
    """Lowered spin limit and one unpublished tile for the duration."""

    def __init__(self, stage, tile, limit=2000):
        self.stage, self.tile, self.limit = stage, tile, limit

    def __enter__(self):
        _C.test_set_spin_limit(self.limit)
        _C.test_unpublished_tile(self.stage, self.tile)
        return self

    def __exit__(self, *exc):
        _C.test_unpublished_tile(self.stage, -1)
        _C.test_set_spin_limit(0)
        _C.set_error_check(False)
        torch.cuda.synchronize()


def _cumsum(host, exclusive=False):
    inc = np.cumsum(host, dtype=np.uint64).astype(np.uint32)
    return np.concatenate([[0], inc[:-1]]).astype(np.uint32) if exclusive else inc


def test_scan_wait_runs_out_and_is_reported():
    lib = _lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = 40 * 4096  # 40 scan tiles
    host = np.random.default_rng(1).integers(0, 100, size=n).astype(np.uint32)
    x = torch.from_numpy(host.view(np.int32)).cuda()
    out = torch.empty_like(x)
    scratch = torch.empty(int(lib.w2w_scan_scratch_bytes(n)), dtype=torch.uint8, device="cuda")
    with hooked(STAGE_SCAN, 3):
        # default mode: the call reports its launch, the scratch word the timeout
        assert lib.w2w_scan_u32(x.data_ptr(), out.data_ptr(), n, 0, scratch.data_ptr(), scratch.numel(), stream) == 0
        assert lib.w2w_scratch_error(scratch.data_ptr(), stream) == W2W_ERR_TIMEOUT
        # checked mode: the call itself returns it
        lib.w2w_set_error_check(1)
        assert lib.w2w_scan_u32(x.data_ptr(), out.data_ptr(), n, 0, scratch.data_ptr(), scratch.numel(),
                                stream) == W2W_ERR_TIMEOUT
        lib.w2w_set_error_check(0)
        # the allocation-free scan: its own error query
        assert lib.w2w_scan_u32_noalloc(x.data_ptr(), out.data_ptr(), n, 0, stream) == 0
        assert lib.w2w_scan_noalloc_error(stream) == W2W_ERR_TIMEOUT
        # the torch binding raises
        with pytest.raises(RuntimeError, match="timed out"):
            _C.scan_u32(x, False)
    # clean again, and correct
    assert lib.w2w_scan_u32(x.data_ptr(), out.data_ptr(), n, 0, scratch.data_ptr(), scratch.numel(), stream) == 0
    assert lib.w2w_scratch_error(scratch.data_ptr(), stream) == 0
    assert np.array_equal(out.cpu().numpy().view(np.uint32), _cumsum(host))
    assert lib.w2w_scan_u32_noalloc(x.data_ptr(), out.data_ptr(), n, 0, stream) == 0
    assert lib.w2w_scan_noalloc_error(stream) == 0
    assert np.array_equal(out.cpu().numpy().view(np.uint32), _cumsum(host))


def test_sort_wait_runs_out_and_is_reported():
    n = 12 * 5120  # 12 tiles of 64-bit keys
    keys = np.random.default_rng(2).integers(0, 1 << 40, size=n).astype(np.uint64)
    k = torch.from_numpy(keys.view(np.int64)).cuda()
    v = torch.arange(n, dtype=torch.int32, device="cuda")
    with hooked(STAGE_SORT, 2):
        with pytest.raises(RuntimeError, match="timed out"):
            _C.sort_pairs_u64(k, v, 0, 40)
    ko, vo = _C.sort_pairs_u64(k, v, 0, 40)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(ko.cpu().numpy().view(np.uint64), keys[order])
    assert np.array_equal(vo.cpu().numpy(), order.astype(np.int32))


def _scene(P=8192, S=192):
    arrays = scenes.make_scene(P, seed=4).activate()
    return arrays, camera.orbit_camera(20.0, 10.0, 2.5, S, S)


@pytest.mark.parametrize("binning,queue", [(0, 0), (1, 0), (0, 1)])
def test_render_sort_wait_is_reported_by_the_deferred_check(binning, queue):
    """The render's sort with its first tile unpublished: the radix sort of
    the emitted keys (binning 0), or the depth sort of the 8192 Gaussians
    (binning 1; two onesweep tiles per pass).  With queue = 1 the persistent
    blend then walks the inconsistent list (stray ids gather a valid row and
    are never blended) and the next render is clean."""
    arrays, cam = _scene()
    with gh.tuned(binning=binning, blend_queue=queue):
        clean = gh.forward(arrays, cam)
        assert clean["num_rendered"] > 2 * 6144
        with hooked(STAGE_SORT, 0):
            gh.forward(arrays, cam)  # returns; its point list is invalid
            with pytest.raises(RuntimeError, match="timed out"):
                _C.check_device_errors()
        again = gh.forward(arrays, cam)
        _C.check_device_errors()
    for key in ("keys", "point_list", "ranges", "n_contrib", "color", "alpha"):
        assert np.array_equal(again[key], clean[key]), key


def test_projection_scan_wait_raises_at_once():
    arrays, cam = _scene()
    clean = gh.forward(arrays, cam)
    with hooked(STAGE_PREPROCESS, 2):
        with pytest.raises(RuntimeError, match="timed out"):
            gh.forward(arrays, cam)
    again = gh.forward(arrays, cam)
    for key in ("offsets", "keys", "point_list", "color"):
        assert np.array_equal(again[key], clean[key]), key
