"""Hierarchical stage timer with the reference's API and stage names
(``jax_qc/profiling/timer.py:40-172``): ``StageTimer.stage(name, fp_type)``
nests, repeated stages aggregate, and ``optional_stage`` is a no-op without a
timer.  Device work is synchronized at stage boundaries with
``torch.cuda.synchronize`` (the reference used ``jax.effects_barrier``)."""

from __future__ import annotations

import time
from contextlib import contextmanager
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import torch


@dataclass
class StageRecord:
    name: str
    wall_time: float = 0.0
    call_count: int = 0
    children: Dict[str, "StageRecord"] = field(default_factory=dict)
    fp_abstraction: str = ""

    def to_dict(self) -> dict:
        return {
            "name": self.name,
            "wall_time": self.wall_time,
            "call_count": self.call_count,
            "fp_abstraction": self.fp_abstraction,
            "children": {k: v.to_dict() for k, v in self.children.items()},
        }


def _sync():
    if torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.synchronize()


class StageTimer:
    def __init__(self, sync_device: bool = True) -> None:
        self.root = StageRecord(name="total")
        self._stack: List[StageRecord] = [self.root]
        self._sync = sync_device

    @contextmanager
    def stage(self, name: str, fp_type: str = ""):
        parent = self._stack[-1]
        rec = parent.children.get(name)
        if rec is None:
            rec = StageRecord(name=name, fp_abstraction=fp_type)
            parent.children[name] = rec
        elif fp_type and not rec.fp_abstraction:
            rec.fp_abstraction = fp_type
        if self._sync:
            _sync()
        t0 = time.perf_counter()
        self._stack.append(rec)
        try:
            yield rec
        finally:
            if self._sync:
                _sync()
            rec.wall_time += time.perf_counter() - t0
            rec.call_count += 1
            self._stack.pop()

    def to_dict(self) -> dict:
        return self.root.to_dict()

    def get(self, *path: str) -> Optional[StageRecord]:
        rec = self.root
        for p in path:
            rec = rec.children.get(p)
            if rec is None:
                return None
        return rec


@contextmanager
def optional_stage(timer: Optional[StageTimer], name: str, fp_type: str = ""):
    if timer is None:
        yield None
    else:
        with timer.stage(name, fp_type) as rec:
            yield rec
