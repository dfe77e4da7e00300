"""Serving loop: render + backward requests over device-resident scenes,
admitted under an HBM budget and batched as they arrive.

A request is (scene, views, upstream image gradients).  Scenes stay resident
on the device.  The loop is continuous batching over a few execution slots,
each with its own CUDA stream and its own grow-only workspace: whenever a slot
is free, every request that has arrived and fits the memory the in-flight
batches leave of the budget joins one batch (one BatchRenderer forward +
backward over all their views), launched on that slot's stream while the
other slots' batches are still running.  So requests that arrive while others
are on the GPU start as soon as a slot and memory free up, and their kernels
overlap on the device with the batches already there; completion is seen by
polling each batch's end event, never by a device-wide synchronisation.
Each request's result is what it would get alone: its images are
bit-identical and its gradients equal up to float atomic order
(tests/test_serve.py).  Latency is arrival to completion, with start and
completion taken from the batch's CUDA events on its stream.

The reference has no serving loop; its per-call path is one
``Renderer.render`` per view (here: one single-view call at a time, FIFO,
``serve_plain``) and stands beside this as the baseline.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .batch import BatchRenderer, View

# per-element and per-instance state bytes of a batched call (geometry state,
# gradients, binning state) used for admission; instances per element are
# estimated from the resolution (about 12 per element at 512^2 for compact
# scenes, scaling with the pixel count)
ELEM_BYTES = 1100
INST_BYTES = 24
PIX_BYTES = 48


@dataclass
class Request:
    rid: int
    scene: int
    cameras: list            # Camera per view
    grads: list              # [3,H,W] upstream gradient per view (device)
    arrival: float = 0.0     # seconds from the start of the run
    # filled by the server
    start: float = 0.0
    done: float = 0.0
    color: list = field(default_factory=list)
    scene_grads: dict = field(default_factory=dict)

    def views(self):
        return [View(self.scene, c) for c in self.cameras]


def request_bytes(req: Request, scenes) -> int:
    P = scenes[req.scene].P
    total = 0
    for c in req.cameras:
        pix = int(c.width) * int(c.height)
        inst = 12.0 * P * pix / (512 * 512)
        total += ELEM_BYTES * P + INST_BYTES * inst + PIX_BYTES * pix
    return int(total)


class _Slot:
    """One execution slot: a stream, a renderer with its own workspace, and
    the batch in flight on it (with its start / end events)."""

    def __init__(self, device, grad_mode):
        self.renderer = BatchRenderer(grad_mode=grad_mode, reuse_buffers=True, device=device)
        self.stream = torch.cuda.Stream(device=device)
        self.batch = None
        self.bytes = 0.0
        self.ev_start = None
        self.ev_end = None


class Server:
    """Continuous-batching request loop over resident scenes."""

    def __init__(self, scenes, hbm_budget_bytes: float = 150e9, max_instances: float = 4e8,
                 max_batch_work: float = 2e7, grad_mode: str = "reference", keep_results: bool = False,
                 slots: int = 2):
        self.scenes = scenes
        self.budget = float(hbm_budget_bytes)
        self.max_instances = float(max_instances)  # keeps a batch's instance count far below the 2^30 limit
        # latency bound: Gaussian-views per batch (sum of P over its views).
        # A batch's time is close to linear in it (about 2.5 ns each on a B200
        # for 256-1024^2 views), so 2e7 keeps a batch near 50 ms and a request
        # that arrives during one waits at most that long before its own.
        self.max_work = float(max_batch_work)
        # every slot keeps one grow-only workspace for its batches: no
        # allocator calls once it has grown to the largest batch (a request's
        # gradients are therefore valid until its slot's next batch unless
        # keep_results copies them)
        dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else None
        self.grad_mode = grad_mode
        self.slots = [_Slot(dev, grad_mode) for _ in range(max(1, int(slots)))] if dev is not None else []
        self.keep = keep_results
        self.batch_ms = []
        self.batch_log = []  # (device start s, device end s, request ids) per completed batch

    @property
    def renderer(self):
        return self.slots[0].renderer

    def workspace_bytes(self) -> int:
        return sum(s.renderer.ws.bytes for s in self.slots)

    def workspace_growths(self) -> int:
        return sum(s.renderer.ws.grown for s in self.slots)

    def release_workspaces(self):
        for s in self.slots:
            s.renderer.ws.bufs.clear()

    def _admit(self, queue, budget=None, at_least_one=True):
        """Requests (in arrival order) that fit the memory budget, the
        instance bound and the work bound of one batch; at least one when
        ``at_least_one`` (nothing else in flight), else possibly none."""
        budget = self.budget if budget is None else budget
        batch, mem, inst, work = [], 0.0, 0.0, 0.0
        for r in queue:
            b = request_bytes(r, self.scenes)
            P = self.scenes[r.scene].P
            i = sum(12.0 * P * c.width * c.height / (512 * 512) for c in r.cameras)
            w = float(P) * len(r.cameras)
            if (batch or not at_least_one) and (mem + b > budget or inst + i > self.max_instances or
                                                work + w > self.max_work):
                break
            batch.append(r)
            mem += b
            inst += i
            work += w
        return batch

    def run_batch(self, batch, renderer=None):
        renderer = self.renderer if renderer is None else renderer
        views = [v for r in batch for v in r.views()]
        grads = [g for r in batch for g in r.grads]
        groups = [k for k, r in enumerate(batch) for _ in r.cameras]
        res = renderer.forward(self.scenes, views)
        out = renderer.backward(res, grads, per_element=self.keep, groups=groups)
        k = 0
        for j, r in enumerate(batch):  # each request: its scene's gradient summed over its views
            r.scene_grads = {name: out[name][j] for name in ("means3D", "opacities", "scales", "rotations", "shs")}
            if self.keep:
                r.scene_grads = {name: g.clone() for name, g in r.scene_grads.items()}
                n = len(r.cameras)
                r.color = [c.clone() for c in res.color[k:k + n]]
                r.scene_grads["per_item"] = [tuple(x.clone() for x in item) for item in out["per_item"][k:k + n]]
                k += n
        return res, out

    def _launch(self, slot, batch, origin):
        slot.stream.wait_stream(torch.cuda.current_stream(slot.stream.device))  # the requests' inputs
        with torch.cuda.stream(slot.stream):
            slot.ev_start = torch.cuda.Event(enable_timing=True)
            slot.ev_start.record(slot.stream)
            self.run_batch(batch, slot.renderer)
            slot.ev_end = torch.cuda.Event(enable_timing=True)
            slot.ev_end.record(slot.stream)
        slot.batch = batch
        slot.bytes = float(sum(request_bytes(r, self.scenes) for r in batch))

    def _complete(self, slot, origin):
        start = origin.elapsed_time(slot.ev_start) / 1e3
        end = origin.elapsed_time(slot.ev_end) / 1e3
        for r in slot.batch:
            r.start, r.done = start, end
        self.batch_ms.append((end - start) * 1e3)
        self.batch_log.append((start, end, [r.rid for r in slot.batch]))
        slot.batch, slot.bytes = None, 0.0

    def serve(self, requests, realtime: bool = True):
        """Process requests (sorted by arrival).  With realtime, arrivals are
        honoured against the wall clock (the loop waits for the next arrival
        when idle); otherwise all requests are present at time 0."""
        pending = sorted(requests, key=lambda r: r.arrival)
        queue = []
        origin = torch.cuda.Event(enable_timing=True)
        origin.record()
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        batches = 0
        while pending or queue or any(s.batch is not None for s in self.slots):
            t = now()
            while pending and (not realtime or pending[0].arrival <= t):
                queue.append(pending.pop(0))
            progressed = False
            for s in self.slots:
                if s.batch is not None and s.ev_end.query():
                    self._complete(s, origin)
                    progressed = True
            free = [s for s in self.slots if s.batch is None]
            if queue and free:
                busy = [s for s in self.slots if s.batch is not None]
                batch = self._admit(queue, self.budget - sum(s.bytes for s in busy), at_least_one=not busy)
                if batch:
                    queue = queue[len(batch):]
                    self._launch(free[0], batch, origin)
                    batches += 1
                    progressed = True
            if not progressed:
                if any(s.batch is not None for s in self.slots) or queue:
                    time.sleep(0.0001)  # a batch is running: poll its end event again shortly
                elif pending:
                    time.sleep(max(0.0, min(pending[0].arrival - now(), 0.001)))
        return dict(batches=batches, wall=now())

    def serve_plain(self, requests, realtime: bool = True):
        """Baseline: one single-view call per view, one request at a time,
        FIFO; each request's gradients are summed over its views, as the
        batched loop returns them."""
        from . import _C
        pending = sorted(requests, key=lambda r: r.arrival)
        dev = self.renderer.device
        bg = torch.ones(3, device=dev)
        empty = torch.empty(0, device=dev)
        gm = self.renderer.grad_mode
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        for r in pending:
            if realtime and r.arrival > now():
                time.sleep(r.arrival - now())
            r.start = now()
            sc = self.scenes[r.scene]
            sums = None
            for c, g in zip(r.cameras, r.grads):
                tt = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev)
                V, Pm, C = tt(c.viewmatrix), tt(c.projmatrix), tt(c.campos)
                R, color, depth, alpha, radii, geom, binb, img = _C.rasterize_gaussians(
                    sc.shs, c.focal_y, sc.scales, sc.means3D, Pm, sc.sh_degree, sc.opacities, sc.rotations, C, V,
                    c.focal_x, c.height, c.width, bg, True)
                z = torch.zeros(1, c.height, c.width, device=dev)
                out = _C.rasterize_gaussians_backward(bg, sc.means3D, radii, empty, sc.scales, sc.rotations, 1.0,
                                                      empty, V, Pm, c.tanfovx, c.tanfovy, g, z, z, sc.shs,
                                                      sc.sh_degree, C, geom, R, binb, img, alpha, False, gm)
                grads = (out[3], out[2], out[6], out[7], out[5])  # means3D, opacities, scales, rotations, shs
                if sums is None:
                    sums = list(grads)
                else:
                    for acc, gr in zip(sums, grads):
                        acc.add_(gr)
            if self.keep:
                r.scene_grads = dict(zip(("means3D", "opacities", "scales", "rotations", "shs"), sums))
            torch.cuda.synchronize()
            r.done = now()
        return dict(wall=now())


def overlapping_batches(batch_log) -> int:
    """Batches that started on the device before the previous one (in start
    order) had finished there."""
    log = sorted(batch_log)
    return sum(1 for a, b in zip(log, log[1:]) if b[0] < a[1])


def latency_stats(requests):
    lat = np.array([r.done - r.arrival for r in requests]) * 1e3
    views = sum(len(r.cameras) for r in requests)
    span = max(r.done for r in requests) - min(r.arrival for r in requests)
    return {"p50_ms": round(float(np.percentile(lat, 50)), 3), "p95_ms": round(float(np.percentile(lat, 95)), 3),
            "p99_ms": round(float(np.percentile(lat, 99)), 3), "mean_ms": round(float(lat.mean()), 3),
            "requests": len(requests), "views": views, "views_per_s": round(views / span, 3),
            "requests_per_s": round(len(requests) / span, 3)}


def poisson_requests(n, rate, scenes, seed=0, device="cuda", views=(1, 8), res=(256, 512, 1024)):
    """n requests with Poisson arrivals at `rate` per second over the resident
    scenes: 1-8 orbit views each at a resolution from `res`, N(0,1) upstream
    gradients."""
    from .camera import orbit_camera
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=n)
    arrivals = np.cumsum(gaps) - gaps[0]
    gen = torch.Generator(device=device).manual_seed(seed + 1)
    out = []
    for k in range(n):
        s = int(rng.integers(len(scenes)))
        nv = int(rng.integers(views[0], views[1] + 1))
        r = int(rng.choice(res))
        cams = [orbit_camera(float(rng.uniform(0, 360)), float(rng.uniform(-30, 30)), 2.5, r, r) for _ in range(nv)]
        grads = [torch.randn(3, r, r, device=device, generator=gen) for _ in range(nv)]
        out.append(Request(k, s, cams, grads, float(arrivals[k])))
    return out
