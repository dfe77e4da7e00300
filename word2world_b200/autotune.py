"""Launch-shape autotuner: picks the library's tuning knobs (blend CTA shape,
per-tile or persistent queue-fed blend, the blend's batch staging (registers
or cp.async), how many heavy tiles the per-pixel backward splits and into how
many segments, radix or depth-ordered binning, the projection pass's register
budget) for a workload by timing it, and remembers the choice per shape
bucket.

The reference's launch shapes are constants (pixelGaussiansFull.cu:99-122,
backward.cu:521-665).  Here they are run-time knobs of the C ABI
(``w2w_tune_set``), and none of them changes a result beyond the order of
float atomic additions, so trying them on the caller's own workload is safe.

Search: coordinate descent over the knobs, starting from the current values;
each candidate runs ``step`` (one forward + backward of the workload) after a
warm-up, timed with CUDA events on the current stream, median of ``reps``.  A
knob keeps a new value only when it beats the best so far by more than
``min_gain`` (timing noise), and descent stops when a round changes nothing.
Choices are cached by bucket key (device name, resolution, Gaussian-count
octave, gradient mode), in memory and, when ``path`` is given, in a JSON file.
"""
from __future__ import annotations

import json
import math
import os
import statistics

import torch

from . import _C

CANDIDATES = {
    "blend_warps": [4, 8],
    "backward_split": [0, 2, 4, 8],
    "backward_ways": [2, 3],
    "binning": [0, 1],
    "blend_queue": [0, 1],
    "preprocess_blocks": [4, 3, 2],
    "blend_stage": [1, 0],
}


def bucket_key(width: int, height: int, P: int, grad_mode: str = "reference", device=None) -> str:
    """Shape bucket: device, image size, Gaussian count to the octave, gradient mode."""
    name = torch.cuda.get_device_name(device) if torch.cuda.is_available() else "cpu"
    octave = int(math.floor(math.log2(max(int(P), 1))))
    return f"{name}|{int(width)}x{int(height)}|P2^{octave}|{grad_mode}"


def current() -> dict:
    """The tuned launch-shape knobs (the library's other switches, such as
    planned_forward, are set with apply but not tuned)."""
    return {k: v for k, v in _C.tune_knobs().items() if k in CANDIDATES}


def apply(knobs: dict) -> dict:
    """Set knobs; returns the previous values of those set."""
    return {k: int(_C.tune_set(k, int(v))) for k, v in knobs.items()}


class Autotuner:
    def __init__(self, path: str | None = None, reps: int = 5, warmup: int = 2, min_gain: float = 0.01,
                 timer=None):
        self.path = path
        self.reps, self.warmup, self.min_gain = int(reps), int(warmup), float(min_gain)
        self.cache: dict = {}
        self.log: list = []
        self._timer = timer or self._cuda_time
        if path and os.path.exists(path):
            with open(path) as f:
                self.cache = json.load(f)

    def _cuda_time(self, step) -> float:
        for _ in range(self.warmup):
            step()
        torch.cuda.synchronize()
        stream = torch.cuda.current_stream()
        times = []
        for _ in range(self.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        return statistics.median(times)

    def _save(self):
        if self.path:
            tmp = self.path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.cache, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)

    def tune(self, key: str, step, candidates: dict | None = None, rounds: int = 2) -> dict:
        """Coordinate descent for bucket ``key``; applies and returns the best
        knobs (with the timings in ``self.log``)."""
        cands = candidates or CANDIDATES
        best = {k: v for k, v in current().items() if k in cands}
        apply(best)
        best_ms = self._timer(step)
        self.log.append((dict(best), best_ms))
        for _ in range(rounds):
            changed = False
            for knob, values in cands.items():
                for v in values:
                    if v == best[knob]:
                        continue
                    trial = dict(best, **{knob: v})
                    apply(trial)
                    ms = self._timer(step)
                    self.log.append((dict(trial), ms))
                    if ms < best_ms * (1.0 - self.min_gain):
                        best, best_ms, changed = trial, ms, True
                apply(best)
            if not changed:
                break
        apply(best)
        self.cache[key] = dict(best, ms=round(best_ms, 4))
        self._save()
        return dict(best)

    def ensure(self, key: str, step, candidates: dict | None = None) -> dict:
        """The cached choice for ``key`` (applied), tuning it first if unknown."""
        if key in self.cache:
            knobs = {k: v for k, v in self.cache[key].items() if k in (candidates or CANDIDATES)}
            apply(knobs)
            return knobs
        return self.tune(key, step, candidates)
