"""The allocation-free scan entry point (w2w_scan_u32_noalloc) agrees with
the scratch-taking one (w2w_scan_u32) on two calls in a row.

It serves callers that cannot allocate device memory or pass scratch (hosts
whose device memory belongs to another allocator, allocation-free loops):
its scratch is a fixed array inside the library.  Called through the C ABI
with ctypes, on torch's current stream.  Kept in its own file, collected
last.
"""
import ctypes
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "word2world_b200", "libw2w_raster.so")
MAX_N = 1 << 24  # W2W_SCAN_NOALLOC_MAX


def _lib():
    lib = ctypes.CDLL(LIB)
    vp, ll, sz = ctypes.c_void_p, ctypes.c_longlong, ctypes.c_size_t
    lib.w2w_scan_u32.argtypes = [vp, vp, ll, ctypes.c_int, vp, sz, vp]
    lib.w2w_scan_u32_noalloc.argtypes = [vp, vp, ll, ctypes.c_int, vp]
    lib.w2w_scan_scratch_bytes.argtypes = [ll]
    lib.w2w_scan_scratch_bytes.restype = sz
    lib.w2w_scan_noalloc_error.argtypes = [vp]
    return lib


def _cumsum(host, exclusive):
    inc = np.cumsum(host, dtype=np.uint64).astype(np.uint32)
    return np.concatenate([[0], inc[:-1]]).astype(np.uint32) if exclusive else inc


def test_noalloc_scan_matches_scratch_entry_point():
    lib = _lib()
    torch.cuda.init()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(7)
    cases = [(3_000_001, 0), (MAX_N, 1)]  # two calls in a row, the second at the maximum size
    for n, exclusive in cases:
        x = torch.from_numpy(rng.poisson(8.0, size=n).astype(np.uint32).view(np.int32)).cuda()
        expect = torch.empty_like(x)
        scratch = torch.empty(int(lib.w2w_scan_scratch_bytes(n)), dtype=torch.uint8, device="cuda")
        assert lib.w2w_scan_u32(x.data_ptr(), expect.data_ptr(), n, exclusive, scratch.data_ptr(), scratch.numel(),
                                stream) == 0
        got = torch.full_like(x, -1)
        assert lib.w2w_scan_u32_noalloc(x.data_ptr(), got.data_ptr(), n, exclusive, stream) == 0
        torch.cuda.synchronize()
        assert torch.equal(got, expect)
        assert np.array_equal(got.cpu().numpy().view(np.uint32), _cumsum(x.cpu().numpy().view(np.uint32), exclusive))
    assert lib.w2w_scan_noalloc_error(stream) == 0


def test_noalloc_scan_back_to_back_after_a_larger_call():
    """Calls queued on one stream with no synchronisation between them, the
    first at the maximum size: each later, smaller call must clear the shared
    array's words it uses, whatever the larger call left beyond them."""
    lib = _lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(11)
    sizes = [MAX_N, 1, 4096, 4097, 12289, 1]  # 4096 elements per scan tile
    xs, outs = [], []
    for k, n in enumerate(sizes):
        x = torch.from_numpy(rng.integers(0, 1 << 20, size=n).astype(np.uint32).view(np.int32)).cuda()
        out = torch.full_like(x, -1)
        assert lib.w2w_scan_u32_noalloc(x.data_ptr(), out.data_ptr(), n, k % 2, stream) == 0
        xs.append(x)
        outs.append(out)
    torch.cuda.synchronize()
    assert lib.w2w_scan_noalloc_error(stream) == 0
    for k, (x, out) in enumerate(zip(xs, outs)):
        assert np.array_equal(out.cpu().numpy().view(np.uint32), _cumsum(x.cpu().numpy().view(np.uint32), k % 2)), k


def test_noalloc_scan_rejects_oversize():
    lib = _lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    x = torch.zeros(16, dtype=torch.int32, device="cuda")
    # the size check comes first: nothing is read or written for n > max
    assert lib.w2w_scan_u32_noalloc(x.data_ptr(), x.data_ptr(), MAX_N + 1, 0, stream) == 3
