"""Sort, scan and tile-range stages vs numpy / the oracle, bit-exact.

Sort distributions follow the reference's sort harnesses
(sorting-optimizations/profile_*_vs_cub.cu: random 64-bit, sorted, reverse,
few unique, sparse high bits, limited range) plus the rasterizer's own
(tile | depth) keys; the oracle is a stable sort on (key, input position).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

from word2world_b200 import _C, scenes  # noqa: E402


def _sort(keys, vals, begin=0, end=64):
    kd, vd = _C.sort_pairs_u64(torch.from_numpy(keys.view(np.int64)).cuda(),
                               torch.from_numpy(vals.view(np.int32)).cuda(), begin, end)
    return kd.cpu().numpy().view(np.uint64), vd.cpu().numpy().view(np.uint32)


def _expect(keys, vals, begin=0, end=64):
    mask = np.uint64((1 << (end - begin)) - 1) if end - begin < 64 else np.uint64(0xFFFFFFFFFFFFFFFF)
    sub = (keys >> np.uint64(begin)) & mask
    order = np.argsort(sub, kind="stable")
    return keys[order], vals[order]


def _dist(kind, n, rng):
    if kind == "random":
        return rng.integers(0, 2**63, size=n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=n, dtype=np.uint64)
    if kind == "sorted":
        return np.sort(rng.integers(0, 2**62, size=n, dtype=np.uint64))
    if kind == "reverse":
        return np.sort(rng.integers(0, 2**62, size=n, dtype=np.uint64))[::-1].copy()
    if kind == "few_unique":
        return rng.choice(np.array([3, 77, 1 << 40, (1 << 63) + 5], dtype=np.uint64), size=n)
    if kind == "high_bits":
        return rng.integers(0, 256, size=n, dtype=np.uint64) << np.uint64(56)
    if kind == "limited":
        return rng.integers(0, 1000, size=n, dtype=np.uint64)
    if kind == "equal":
        return np.full(n, 12345, dtype=np.uint64)
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["random", "sorted", "reverse", "few_unique", "high_bits", "limited", "equal"])
@pytest.mark.parametrize("n", [1, 1000, 4096, 4097, 20000])
def test_sort_distributions(kind, n):
    rng = np.random.default_rng(42 + n)
    keys = _dist(kind, n, rng)
    vals = np.arange(n, dtype=np.uint32)
    k, v = _sort(keys, vals)
    ek, ev = _expect(keys, vals)
    assert np.array_equal(k, ek) and np.array_equal(v, ev)


def test_sort_empty():
    k, v = _sort(np.zeros(0, np.uint64), np.zeros(0, np.uint32))
    assert k.size == 0 and v.size == 0


@pytest.mark.parametrize("begin,end", [(0, 44), (32, 44), (8, 24), (0, 0), (60, 64)])
def test_sort_bit_ranges(begin, end):
    keys, vals = scenes.sort_workload(50000, seed=begin + end)
    k, v = _sort(keys, vals, begin, end)
    ek, ev = _expect(keys, vals, begin, end)
    assert np.array_equal(k, ek) and np.array_equal(v, ev)


def test_sort_rasterizer_keys_2m():
    keys, vals = scenes.sort_workload(2_000_000, seed=1)
    k, v = _sort(keys, vals, 0, 44)
    ek, ev = _expect(keys, vals, 0, 44)
    assert np.array_equal(k, ek) and np.array_equal(v, ev)


@pytest.mark.slow
def test_sort_20m_properties():
    """The isolated-stage size: 20M keys.  Checked by size-independent
    properties (sorted, permutation of the input, stable) instead of a CPU sort."""
    keys, vals = scenes.sort_workload(20_000_000, seed=2)
    k, v = _sort(keys, vals, 0, 44)
    assert np.all(k[1:] >= k[:-1])
    assert np.array_equal(keys[v], k)          # values are input positions: a permutation carrying the keys
    same = k[1:] == k[:-1]
    assert np.all(v[1:][same] > v[:-1][same])  # stability: equal keys keep input order
    assert np.array_equal(np.sort(v), np.arange(len(v), dtype=np.uint32))


@pytest.mark.parametrize("n", [1, 31, 4096, 4097, 100000, 2_000_000])
@pytest.mark.parametrize("exclusive", [False, True])
def test_scan(n, exclusive):
    x = scenes.scan_workload(n, seed=n)
    out = _C.scan_u32(torch.from_numpy(x.view(np.int32)).cuda(), exclusive).cpu().numpy().view(np.uint32)
    inc = np.cumsum(x, dtype=np.uint64).astype(np.uint32)
    exp = np.concatenate([[0], inc[:-1]]).astype(np.uint32) if exclusive else inc
    assert np.array_equal(out, exp)


def test_tile_ranges():
    import oracle
    keys, vals = scenes.sort_workload(100000, seed=3, num_tiles=1024)
    keys = np.sort(keys)
    got = _C.tile_ranges(torch.from_numpy(keys.view(np.int64)).cuda(), 32, 1024).cpu().numpy().view(np.uint32)
    exp = np.zeros((1024, 2), np.uint32)
    oracle.lib().orc_tile_ranges(oracle._p(keys), oracle.ctypes.c_longlong(len(keys)), oracle._p(exp),
                                 oracle.ctypes.c_int(1024))
    assert np.array_equal(got, exp)
