"""Serving loop: admission under the memory budget (CPU), and each request's
result the same alone and inside a mixed batch (GPU)."""
from types import SimpleNamespace

import numpy as np
import pytest

torch = pytest.importorskip("torch")

try:
    from word2world_b200 import serve as sv
except ImportError:  # the extension is not built here
    sv = None


def _fake_req(rid, scene, res, nv):
    cam = SimpleNamespace(width=res, height=res)
    return SimpleNamespace(rid=rid, scene=scene, cameras=[cam] * nv)


@pytest.mark.skipif(sv is None, reason="extension not built")
def test_admission_respects_budget():
    scenes = [SimpleNamespace(P=100_000), SimpleNamespace(P=10_000)]
    srv = sv.Server.__new__(sv.Server)
    srv.scenes, srv.max_instances, srv.max_work = scenes, 1e12, 1e12
    q = [_fake_req(0, 0, 512, 4), _fake_req(1, 1, 256, 1), _fake_req(2, 0, 1024, 8)]
    sizes = [sv.request_bytes(r, scenes) for r in q]
    srv.budget = sizes[0] + sizes[1] + 1
    assert [r.rid for r in srv._admit(q)] == [0, 1]
    srv.budget = 1.0  # a single oversized request is still admitted alone
    assert [r.rid for r in srv._admit(q)] == [0]
    srv.budget, srv.max_work = 1e15, 4 * 100_000 + 10_000  # the work bound: Gaussian-views per batch
    assert [r.rid for r in srv._admit(q)] == [0, 1]


@pytest.mark.skipif(sv is None, reason="extension not built")
def test_workspace_grows_only_when_needed():
    from word2world_b200.batch import _Workspace
    ws = _Workspace(torch.device("cpu"))
    a = ws.f32("g", 100, 3)
    assert a.shape == (100, 3) and ws.grown == 1
    b = ws.f32("g", 190, 3)  # within the 2x headroom: same storage
    assert b.shape == (190, 3) and ws.grown == 1 and b.data_ptr() == a.data_ptr()
    c = ws.f32("g", 1000, 3)
    assert c.shape == (1000, 3) and ws.grown == 2
    assert ws.f32("g", 0, 3).shape == (0, 3) and ws.i64("idx", 0).numel() == 0
    assert ws.take("u", 7).numel() == 7 and ws.bytes % 256 == 0


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")
def test_request_same_alone_and_in_the_mix():
    import parity
    from word2world_b200 import scenes as S
    from word2world_b200.batch import Scene
    scs = [Scene.from_arrays(S.make_scene(P, seed=20 + k, layout="ball").activate(), "cuda")
           for k, P in enumerate((4000, 9000, 2500))]
    reqs = sv.poisson_requests(10, rate=1000.0, scenes=scs, seed=5, views=(1, 3), res=(64, 96, 128))
    srv = sv.Server(scs, keep_results=True)
    srv.serve(reqs, realtime=False)
    for r in (reqs[0], reqs[4], reqs[9]):
        mixed_color, mixed_grads = r.color, r.scene_grads["per_item"]
        alone = sv.Request(r.rid, r.scene, r.cameras, r.grads)
        srv.run_batch([alone])
        torch.cuda.synchronize()
        for a, b in zip(alone.color, mixed_color):
            assert parity.bit_mismatch(a.cpu().numpy(), b.cpu().numpy()) == 0
        for ga, gb in zip(alone.scene_grads["per_item"], mixed_grads):
            for name, x, y in zip(parity.GRAD_NAMES, ga, gb):
                chk = parity.grad_check(x.cpu().numpy(), y.cpu().numpy(), row_rtol=parity.SAME_IMPL_ROW_RTOL)
                assert chk["norm_rel"] <= 1e-5 and chk["n_bad"] == 0, (r.rid, name, chk)
    st = sv.latency_stats(reqs)
    assert st["requests"] == 10 and st["p99_ms"] >= st["p50_ms"] > 0
    # the same stream again: the workspace already holds the largest batch
    grown = srv.workspace_growths()
    srv.serve(sv.poisson_requests(10, rate=1000.0, scenes=scs, seed=5, views=(1, 3), res=(64, 96, 128)),
              realtime=False)
    assert srv.workspace_growths() == grown


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")
def test_batches_overlap_on_the_device():
    """With two slots, a batch admitted while another is running starts on the
    device before that one ends (CUDA events on the slots' streams), and the
    overlapped results equal each request run alone."""
    import parity
    from word2world_b200 import scenes as S
    from word2world_b200.batch import Scene
    # batches of several milliseconds of device work (the host issues one in
    # about a millisecond, so smaller ones would finish before the next starts)
    scs = [Scene.from_arrays(S.make_scene(P, seed=40 + k, layout="ball").activate(), "cuda")
           for k, P in enumerate((400000, 300000))]
    # at most one request per batch (the work bound holds one request of the
    # larger scene): eight batches through two slots.  A first pass grows both
    # slots' workspaces (a growth returns memory to the driver, which
    # synchronises the device); the second runs as a warmed-up server does.
    srv = sv.Server(scs, keep_results=True, max_batch_work=1.7e6, slots=2)
    srv.serve(sv.poisson_requests(8, rate=1000.0, scenes=scs, seed=9, views=(4, 4), res=(512,)), realtime=False)
    srv.batch_log = []
    reqs = sv.poisson_requests(8, rate=1000.0, scenes=scs, seed=9, views=(4, 4), res=(512,))
    info = srv.serve(reqs, realtime=False)
    assert info["batches"] == 8 and len(srv.batch_log) == 8
    assert sv.overlapping_batches(srv.batch_log) >= 1, srv.batch_log
    for r in reqs:
        assert r.done > r.start >= 0.0
    for r in (reqs[1], reqs[6]):
        alone = sv.Request(r.rid, r.scene, r.cameras, r.grads)
        srv.run_batch([alone])
        torch.cuda.synchronize()
        for a, b in zip(alone.color, r.color):
            assert parity.bit_mismatch(a.cpu().numpy(), b.cpu().numpy()) == 0
        for ga, gb in zip(alone.scene_grads["per_item"], r.scene_grads["per_item"]):
            for name, x, y in zip(parity.GRAD_NAMES, ga, gb):
                # 400k-Gaussian views: a handful of elements may fall outside
                # the row-relative bound through atomic order alone
                chk = parity.grad_check(x.cpu().numpy(), y.cpu().numpy(), row_rtol=parity.SAME_IMPL_ROW_RTOL)
                assert chk["norm_rel"] <= 1e-5 and chk["n_bad"] <= chk["n"] // 100000, (r.rid, name, chk)
