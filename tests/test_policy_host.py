"""Host logic of the mixed-precision policy (CPU only): which precision and
density-screening threshold the Fock builder asks the engine for, build by
build, with a recording stand-in for the direct engine."""

from __future__ import annotations

import pytest
import torch

from jax_examples_b200 import fock as fk
from jax_examples_b200.core import CalcConfig


class _Event:
    def __init__(self, **kw):
        pass

    def record(self):
        pass

    def synchronize(self):
        pass

    def elapsed_time(self, other):
        return 0.0


class _RecordingEngine:
    """Has the direct engine's interface; records (precision, dens_tau)."""

    device = torch.device("cpu")
    n_basis = 2

    def __init__(self):
        self.calls = []

    def jk(self, D, precision="fp64", mixed_tau=1e-7, dens_tau=0.0):
        self.calls.append((precision, dens_tau))
        return torch.zeros_like(D), torch.zeros_like(D)


@pytest.fixture(autouse=True)
def _no_cuda_events(monkeypatch):
    monkeypatch.setattr(fk.torch.cuda, "Event", _Event)


def _drive(cfg, errors):
    eng = _RecordingEngine()
    fb = fk.FockBuilder(eng, cfg)
    D = torch.eye(2, dtype=torch.float64)
    fb.jk(D)
    for k, err in enumerate(errors):
        fb.observe(err)
        fb.jk(D * (1.0 + 0.1 * (k + 1)))
    return eng.calls


def test_incremental_mixed_builds_screen_relative_to_the_scf_error():
    cfg = CalcConfig(precision="mixed", incremental=True)
    calls = _drive(cfg, [0.5, 3e-2, 1e-3])
    assert calls[0] == ("mixed", cfg.mixed_full_dens_tau)  # the first build is a full one
    assert calls[1][0] == "mixed" and calls[1][1] == pytest.approx(cfg.mixed_dens_rel * 0.5)
    assert calls[2][1] == pytest.approx(cfg.mixed_dens_rel * 3e-2)
    assert calls[3][1] == pytest.approx(cfg.mixed_dens_tau)  # 1e-9 is below the floor 2e-8


def test_relative_screening_off_and_fp64_switch():
    cfg = CalcConfig(precision="mixed", incremental=True, mixed_dens_rel=0.0)
    calls = _drive(cfg, [0.5, 5e-5, 1e-5])
    assert calls[1] == ("mixed", cfg.mixed_dens_tau)
    # below fp64_switch: a full FP64 build at the switch threshold, then the FP64 tail
    assert calls[2] == ("fp64", cfg.fp64_switch_dens_tau)
    assert calls[3] == ("fp64", cfg.fp64_tail_dens_tau)


def test_plain_fp64_builds_are_unscreened():
    cfg = CalcConfig(precision="fp64", incremental=False)
    calls = _drive(cfg, [0.5, 1e-3])
    assert all(c == ("fp64", 0.0) for c in calls)
