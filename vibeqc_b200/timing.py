"""Device-side stage timer (CUDA events on the current stream)."""

from __future__ import annotations

from collections import defaultdict
from contextlib import contextmanager

import torch


class StageTimer:
    def __init__(self):
        self.enabled = False
        self._events: list = []

    def reset(self) -> None:
        self._events = []

    @contextmanager
    def stage(self, name: str):
        if not self.enabled:
            yield
            return
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record()
        try:
            yield
        finally:
            end.record()
            self._events.append((name, start, end))

    def summary(self) -> dict:
        torch.cuda.synchronize()
        out = defaultdict(float)
        counts = defaultdict(int)
        for name, s, e in self._events:
            out[name] += s.elapsed_time(e)
            counts[name] += 1
        return {k: {"ms": round(v, 3), "launch_groups": counts[k]} for k, v in out.items()}


TIMER = StageTimer()
