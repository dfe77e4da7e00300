"""Two-rank gloo run of the replica path: each rank renders its shard of the
views (with the oracle, on CPU), timings reduce by max over ranks, and the
gathered images equal a single-process render."""
import os

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import oracle
    from word2world_b200 import camera, dist as wd, scenes
    sc = scenes.make_scene(600, seed=2)
    m, o, s, q_, sh = sc.activate()
    views = camera.orbit_views(4, 2.5, 48, 48)
    mine = wd.shard(list(range(4)), rank, world)
    imgs = {}
    for v in mine:
        st = oracle.RasterSettings.from_camera(views[v])
        imgs[v] = oracle.forward(st, m, s, q_, o, sh)["color"]
    t = wd.max_over_ranks(float(rank + 1))
    total = wd.sum_over_ranks(float(len(mine)))
    gathered = [None] * world
    dist.all_gather_object(gathered, imgs)
    if rank == 0:
        allimgs = {}
        for g in gathered:
            allimgs.update(g)
        q.put((t, total, {k: v.tolist() for k, v in allimgs.items()}))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    t, total, imgs = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert t == 2.0 and total == 4.0
    import oracle
    from word2world_b200 import camera, scenes
    sc = scenes.make_scene(600, seed=2)
    m, o, s, q_, sh = sc.activate()
    for v, cam in enumerate(camera.orbit_views(4, 2.5, 48, 48)):
        ref = oracle.forward(oracle.RasterSettings.from_camera(cam), m, s, q_, o, sh)["color"]
        assert np.array_equal(np.asarray(imgs[v], np.float32), ref)


def test_shard_partition():
    from word2world_b200.dist import shard
    items = list(range(10))
    parts = [shard(items, r, 3) for r in range(3)]
    assert sum(parts, []) == items and [len(p) for p in parts] == [4, 3, 3]
