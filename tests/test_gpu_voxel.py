"""Voxel occupancy field (compute_voxel_field.cu:25-124) against the numpy
restatement of the reference kernel and against the reference kernel itself
(built from its source into oracle/_ref), plus the host-pointer entry point,
determinism and edge cases."""
import ctypes
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

from oracle import voxel as ovox  # noqa: E402
from word2world_b200 import voxel  # noqa: E402
from word2world_b200.batch import _LIB_PATH  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "compute_voxel_field.so")


def _gaussians(P, seed):
    rng = np.random.default_rng(seed)
    means = rng.uniform(-1.0, 1.0, size=(P, 3)).astype(np.float32)
    means[: P // 10] = np.round(means[: P // 10] * 4) / 4  # on block boundaries of B = 4, 8
    q = rng.normal(size=(P, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    Rm = np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
                   np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
                   np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)], 1)
    L = Rm * rng.uniform(0.02, 0.15, size=(P, 1, 3))
    S = L @ L.transpose(0, 2, 1)
    covs = np.stack([S[:, 0, 0], S[:, 0, 1], S[:, 0, 2], S[:, 1, 1], S[:, 1, 2], S[:, 2, 2]], 1).astype(np.float32)
    opac = rng.uniform(0.0, 1.0, size=(P, 1)).astype(np.float32)
    return means, covs, opac


def _gpu(means, covs, opac, R, B, relax):
    t = lambda a: torch.from_numpy(a).cuda()
    return voxel.voxel_field(t(means), t(covs), t(opac), R, B, relax).cpu().numpy()


@pytest.mark.parametrize("R,B,relax", [(16, 4, 0.1), (13, 3, 0.0), (12, 2, 0.6)])
def test_matches_restated_reference(R, B, relax):
    means, covs, opac = _gaussians(300, seed=R)
    got = _gpu(means, covs, opac, R, B, relax)
    want = ovox.voxel_field(means, covs, opac, R, B, relax)
    assert got.shape == (R, R, R)
    np.testing.assert_allclose(got, want, rtol=2e-5, atol=1e-6)


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference voxel kernel not built (oracle/build_ref.py)")
def test_matches_reference_kernel():
    means, covs, opac = _gaussians(3000, seed=7)
    R, B, relax = 32, 8, 0.1
    ref = ctypes.CDLL(REF_SO)
    fp = ctypes.POINTER(ctypes.c_float)
    ref.compute_voxel_field_cuda.argtypes = [fp, fp, fp, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float]
    want = np.zeros(R ** 3, np.float32)
    ptr = lambda a: a.ctypes.data_as(fp)
    m, c, o = (np.ascontiguousarray(x) for x in (means, covs, opac))
    ref.compute_voxel_field_cuda(ptr(want), ptr(m), ptr(c), ptr(o), 3000, R, B, relax)
    got = _gpu(means, covs, opac, R, B, relax)
    np.testing.assert_allclose(got.reshape(-1), want, rtol=2e-5, atol=1e-6)
    # and the host-pointer entry point of this library is the device one, bit for bit
    lib = ctypes.CDLL(_LIB_PATH)
    lib.w2w_compute_voxel_field.argtypes = ref.compute_voxel_field_cuda.argtypes
    host = np.zeros(R ** 3, np.float32)
    assert lib.w2w_compute_voxel_field(ptr(host), ptr(m), ptr(c), ptr(o), 3000, R, B, relax) == 0
    assert np.array_equal(host, got.reshape(-1))


def test_deterministic_and_edges():
    means, covs, opac = _gaussians(5000, seed=3)
    a = _gpu(means, covs, opac, 40, 5, 0.1)
    b = _gpu(means, covs, opac, 40, 5, 0.1)
    assert np.array_equal(a, b) and np.isfinite(a).all() and a.max() > 0
    empty = np.zeros((0, 3), np.float32)
    z = _gpu(empty, np.zeros((0, 6), np.float32), np.zeros((0, 1), np.float32), 8, 2, 0.1)
    assert z.shape == (8, 8, 8) and not z.any()
    far = means + 10.0  # outside every block: nothing binned
    assert not _gpu(far, covs, opac, 8, 2, 0.1).any()
    with pytest.raises(RuntimeError):
        _gpu(means, covs, opac, 1, 2, 0.1)


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference voxel kernel not built (oracle/build_ref.py)")
def test_speed_against_reference_kernel():
    """Both host-pointer entry points (allocation, copies and kernel) on a
    64^3 grid over 20k Gaussians; printed, and this one must be faster."""
    import time
    means, covs, opac = _gaussians(20000, seed=11)
    R, B, relax = 64, 8, 0.1
    fp = ctypes.POINTER(ctypes.c_float)
    ptr = lambda a: a.ctypes.data_as(fp)
    m, c, o = (np.ascontiguousarray(x) for x in (means, covs, opac))
    ref = ctypes.CDLL(REF_SO)
    lib = ctypes.CDLL(_LIB_PATH)
    for fn in (ref.compute_voxel_field_cuda, lib.w2w_compute_voxel_field):
        fn.argtypes = [fp, fp, fp, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float]
    out_r, out_w = np.zeros(R ** 3, np.float32), np.zeros(R ** 3, np.float32)

    def best(fn, out):
        ts = []
        for _ in range(10):
            t = time.perf_counter()
            fn(ptr(out), ptr(m), ptr(c), ptr(o), 20000, R, B, relax)
            ts.append(time.perf_counter() - t)
        print(fn.__name__ if hasattr(fn, "__name__") else fn, [round(x * 1e3, 2) for x in ts])
        return min(ts[1:])
    t_ref = best(ref.compute_voxel_field_cuda, out_r)
    t_w2w = best(lib.w2w_compute_voxel_field, out_w)
    np.testing.assert_allclose(out_w, out_r, rtol=2e-5, atol=1e-6)
    print(f"voxel field 64^3, 20k Gaussians: reference {t_ref * 1e3:.2f} ms, this {t_w2w * 1e3:.2f} ms "
          f"({t_ref / t_w2w:.1f}x)")
    assert t_w2w < t_ref
