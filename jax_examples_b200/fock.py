"""Fock builders (``jax_qc/scf/fock.py:31-79``) over the direct engine.

``build_fock_rhf(H, D, ERI)`` and ``build_fock_uhf(H, Da, Db, ERI)`` keep the
reference signatures; ERI may be a :class:`DirectERI` handle (fused kernels,
no N^4 tensor) or a dense (n,n,n,n) tensor (einsum, as the reference).

:class:`FockBuilder` is the stateful builder the SCF drivers use.  It adds
the precision policy of the mixed path:

* ``precision="fp64"``: every build is a full FP64 build (the plain kernel).
* ``precision="mixed"``: quartets with Q_ij Q_kl < ``mixed_tau`` run in FP32
  (FP64 accumulation), and with ``incremental=True`` each build contracts only
  the density change dD = D - D_prev (J, K are linear in D) with density-
  weighted screening, the error of which is reset by a full rebuild every
  ``rebuild_every`` builds of the mixed phase (itself screened at ``mixed_full_dens_tau``, 1e-9:
  8.3 -> 5.6 ms on (H2O)16 with the same iterations and final error).  In
  this phase the incremental builds screen at
  ``mixed_dens_tau``, raised to ``mixed_dens_rel`` times the last SCF error
  while that is larger (the early Fock matrices only steer the next density;
  a factor of 1e-6 saves 4-10% of the Fock time, 1e-5 and more cost erratic
  extra iterations).  When the SCF error
  drops below ``fp64_switch`` the builder switches to FP64 with a full
  rebuild (screened at ``fp64_switch_dens_tau``, unscreened by default; it
  drops the errors of the mixed phase) and then incremental
  FP64 builds screened at ``fp64_tail_dens_tau`` (1e-11: (H2O)16 ends within
  about 1e-7 Eh of the plain FP64 energy; the full rebuild at the switch is
  what keeps it there, without it the mixed-phase errors stay at 1e-5 Eh),
  and convergence is only accepted after ``fp64_tail_iters`` of them: the
  final energy is an FP64 energy.  The SCF drivers clear their DIIS history
  at the switch (``diis_reset_at_switch``): the reported energy uses the
  extrapolated Fock matrix (``rhf.py:80-81``), which would otherwise keep
  mixing in mixed-phase Fock matrices and their FP32 and screening errors
  (up to 1.6e-6 Eh in the 64-cluster sweep).
"""

from __future__ import annotations

import numpy as np
import torch


def _is_direct(ERI) -> bool:
    return hasattr(ERI, "jk") and hasattr(ERI, "n_basis")


def _dense_jk(D, ERI):
    J = torch.einsum("ls,mnls->mn", D, ERI)
    K = torch.einsum("ls,msln->mn", D, ERI)
    return J, K


def _as_dev(x, dev):
    if torch.is_tensor(x):
        return x.to(device=dev, dtype=torch.float64)
    return torch.as_tensor(np.asarray(x), dtype=torch.float64, device=dev)


def coulomb(D, ERI):
    """J_mn = sum_ls D_ls (mn|ls) (``fock.py:31-33``)."""
    if _is_direct(ERI):
        return ERI.jk(D)[0]
    return _dense_jk(D, ERI)[0]


def exchange(D, ERI):
    """K_mn = sum_ls D_ls (ms|ln) (``fock.py:36-38``)."""
    if _is_direct(ERI):
        return ERI.jk(D)[1]
    return _dense_jk(D, ERI)[1]


def build_fock_rhf(H_core, D, ERI):
    """F = H + J - 1/2 K (``fock.py:41-47``)."""
    if _is_direct(ERI):
        dev = ERI.device
        J, K = ERI.jk(_as_dev(D, dev))
        return _as_dev(H_core, dev) + J - 0.5 * K
    J, K = _dense_jk(D, ERI)
    return H_core + J - 0.5 * K


def build_fock_uhf(H_core, D_alpha, D_beta, ERI):
    """F_s = H + J(Da+Db) - K(Ds) (``fock.py:50-79``)."""
    if _is_direct(ERI):
        dev = ERI.device
        J, K = ERI.jk(torch.stack([_as_dev(D_alpha, dev), _as_dev(D_beta, dev)]))
        H = _as_dev(H_core, dev)
        Jt = J[0] + J[1]
        return H + Jt - K[0], H + Jt - K[1]
    Dt = D_alpha + D_beta
    J = _dense_jk(Dt, ERI)[0]
    return H_core + J - _dense_jk(D_alpha, ERI)[1], H_core + J - _dense_jk(D_beta, ERI)[1]


class FockBuilder:
    """Stateful J/K builder implementing the SCF precision policy."""

    def __init__(self, ERI, config, rebuild_every: int = 8, dens_tau: float = 1e-12):
        self.eri = ERI
        self.direct = _is_direct(ERI)
        if self.direct:
            self.device = ERI.device
        else:
            self.device = ERI.device if torch.is_tensor(ERI) else torch.device("cpu")
            if not torch.is_tensor(ERI):
                self.eri = torch.as_tensor(np.asarray(ERI), dtype=torch.float64)
        self.precision = getattr(config, "precision", "fp64")
        self.mixed_tau = float(getattr(config, "mixed_tau", 1e-4))
        self.incremental = bool(getattr(config, "incremental", False)) and self.direct
        self.fp64_tail = int(getattr(config, "fp64_tail_iters", 2))
        self.fp64_switch = float(getattr(config, "fp64_switch", 1e-5))
        self.rebuild_every = rebuild_every
        self.dens_tau = dens_tau
        self.mixed_dens_tau = float(getattr(config, "mixed_dens_tau", 1e-8))
        self.mixed_dens_rel = float(getattr(config, "mixed_dens_rel", 0.0))  # 0: fixed threshold
        self._last_err = None  # max|DIIS error| of the last iteration
        self.tail_dens_tau = float(getattr(config, "fp64_tail_dens_tau", dens_tau))
        self.mixed_full_dens_tau = float(getattr(config, "mixed_full_dens_tau", 0.0))
        self.switch_dens_tau = float(getattr(config, "fp64_switch_dens_tau", 0.0))
        self.phase = "mixed" if (self.precision == "mixed" and self.direct) else "fp64"
        self.fp64_builds_after_switch = 0
        self.switched = self.phase == "fp64"
        self._prev = None  # (D stack, J stack, K stack) of the last build
        self._since_full = 0
        self._events = []  # (start, end) CUDA events of every build
        self._kinds = []  # "<precision>-full" / "<precision>-inc" of every build
        self.log = {"builds_mixed": 0, "builds_fp64": 0, "incremental_builds": 0, "jk_seconds": 0.0}

    # ----------------------------------------------------------------- core
    def _jk_stack(self, Ds):
        D = torch.stack([_as_dev(d, self.device) for d in Ds])
        if not self.direct:
            J = torch.stack([_dense_jk(d, self.eri)[0] for d in D])
            K = torch.stack([_dense_jk(d, self.eri)[1] for d in D])
            self.log["builds_fp64"] += 1
            return J, K
        prec = self.phase
        key = "builds_mixed" if prec == "mixed" else "builds_fp64"
        self.log[key] += 1
        if prec == "fp64":
            self.fp64_builds_after_switch += 1 if self.switched else 0
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        # periodic rebuilds in the mixed phase (and on the plain incremental
        # path); the FP64 tail of the mixed policy has none
        tail = self.precision == "mixed" and prec == "fp64"
        use_inc = self.incremental and self._prev is not None and (tail or self._since_full < self.rebuild_every)
        if use_inc and self._prev[0].shape == D.shape:
            dD = D - self._prev[0]
            if prec == "mixed":
                tau = max(self.mixed_dens_tau, self.dens_tau)
                if self.mixed_dens_rel > 0.0 and self._last_err is not None:
                    tau = max(tau, self.mixed_dens_rel * self._last_err)
            elif self.precision == "mixed":
                tau = max(self.tail_dens_tau, self.dens_tau)  # FP64 tail of the mixed policy
            else:
                tau = self.dens_tau
            dJ, dK = self.eri.jk(dD, precision=prec, mixed_tau=self.mixed_tau, dens_tau=tau)
            J = self._prev[1] + dJ
            K = self._prev[2] + dK
            self._since_full += 1
            self.log["incremental_builds"] += 1
            self._kinds.append(prec + "-inc")
        else:
            if prec == "mixed":
                tau = self.mixed_full_dens_tau
            elif self.precision == "mixed":
                tau = self.switch_dens_tau  # the FP64 rebuild at the switch
            else:
                tau = 0.0  # plain FP64: unscreened, the reference's build
            J, K = self.eri.jk(D, precision=prec, mixed_tau=self.mixed_tau, dens_tau=tau)
            self._since_full = 0
            self._kinds.append(prec + "-full")
        if self.incremental:
            self._prev = (D, J, K)
        e1.record()
        self._events.append((e0, e1))
        return J, K

    def jk(self, D):
        J, K = self._jk_stack([D])
        return J[0], K[0]

    def rhf(self, H, D):
        J, K = self._jk_stack([D])
        return H + J[0] - 0.5 * K[0]

    def uhf(self, H, Da, Db):
        J, K = self._jk_stack([Da, Db])
        Jt = J[0] + J[1]
        return H + Jt - K[0], H + Jt - K[1]

    # --------------------------------------------------------------- policy
    def observe(self, err_max: float) -> bool:
        """Called once per SCF iteration with max|DIIS error|; True when this
        call switched the builder from the mixed phase to FP64."""
        self._last_err = float(err_max)
        if self.phase == "mixed" and err_max < self.fp64_switch:
            self.phase = "fp64"
            self.switched = True
            self._prev = None  # next build is a full FP64 build
            return True
        return False

    def converged_ok(self) -> bool:
        if self.precision != "mixed" or not self.direct:
            return True
        return self.phase == "fp64" and self.fp64_builds_after_switch >= self.fp64_tail

    def record(self) -> dict:
        """Build counters, the device time of all J/K builds (CUDA events) and
        each build's kind and milliseconds."""
        if self._events:
            self._events[-1][1].synchronize()
            ms = [a.elapsed_time(b) for a, b in self._events]
            self.log["jk_seconds"] = sum(ms) * 1e-3
            self.log["build_ms"] = [[k, round(t, 3)] for k, t in zip(self._kinds, ms)]
        return dict(self.log, precision=self.precision, mixed_tau=self.mixed_tau,
                    incremental=self.incremental)
