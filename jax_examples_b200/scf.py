"""RHF / UHF drivers with DIIS, in torch FP64 on the device.

Same algorithm, convergence test and guess as the reference:

* ``run_rhf``  -- ``jax_qc/scf/rhf.py:95-169`` (core guess, Loewdin X,
  F0 from the guess density, loop of ``scf_step_rhf`` ``rhf.py:52-92``,
  converged when dE < conv and max|e| < max(conv, 1e-6)).
* ``run_uhf``  -- ``jax_qc/scf/uhf.py:187-287`` with the alpha-repulsion
  guess of ``scf/guess.py:42-115`` and 0.3 damping for the first 5
  iterations of open-shell systems.
* DIIS       -- ``jax_qc/scf/diis.py:53-199`` (ring buffer that evicts the
  oldest pair, Pulay B-matrix with the singular fallback).

The Fock build goes through :mod:`jax_examples_b200.fock`, i.e. the fused
ERI + J/K kernels when ``ints.ERI`` is a DirectERI handle.  In mixed precision
(``CalcConfig.precision == "mixed"``) the early iterations use the FP32/FP64
split kernel and incremental Fock builds (F from the density change); once
the DIIS error is below ``fp64_switch`` the build returns to FP64 with a full
rebuild, and at least ``fp64_tail_iters`` FP64 iterations run before
convergence is accepted, so the converged energy is an FP64 energy.
"""

from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from .core import CalcConfig, SCFResult, SCFState
from .fock import FockBuilder
from .profiling import StageTimer, optional_stage


def _t(x, dev):
    return torch.as_tensor(np.asarray(x) if not torch.is_tensor(x) else x, dtype=torch.float64, device=dev)


def symmetric_orthogonalization(S: torch.Tensor) -> torch.Tensor:
    """X = S^{-1/2} (``orthogonalize.py:22-26``)."""
    w, U = torch.linalg.eigh(S)
    return (U * (1.0 / torch.sqrt(w))[None, :]) @ U.T


def _diagonalize(F, X):
    e, Cp = torch.linalg.eigh(X.T @ F @ X)
    return e, X @ Cp


def diis_error(F, D, S, X):
    """X^T (F D S - S D F) X (``diis.py:53-59``)."""
    return X.T @ (F @ D @ S - S @ D @ F) @ X


class DIIS:
    """Pulay DIIS ring buffer (``diis.py:26-130``)."""

    def __init__(self, size: int):
        self.size = size
        self.F = []
        self.E = []

    def clear(self) -> None:
        self.F.clear()
        self.E.clear()

    def push(self, F, e):
        self.F.append(F)
        self.E.append(e)
        if len(self.F) > self.size:
            self.F.pop(0)
            self.E.pop(0)

    def extrapolate(self, F, e):
        self.push(F, e)
        m = len(self.F)
        if m < 2:
            return F
        E = torch.stack(self.E).reshape(m, -1)
        B = torch.empty((m + 1, m + 1), dtype=torch.float64, device=F.device)
        B[:m, :m] = E @ E.T
        B[m, :m] = -1.0
        B[:m, m] = -1.0
        B[m, m] = 0.0
        rhs = torch.zeros(m + 1, dtype=torch.float64, device=F.device)
        rhs[m] = -1.0
        Bh = B.cpu().numpy()
        try:
            c = np.linalg.solve(Bh, rhs.cpu().numpy())[:m]
        except np.linalg.LinAlgError:
            return F
        return torch.einsum("i,imn->mn", torch.as_tensor(c, dtype=torch.float64, device=F.device),
                            torch.stack(self.F))


def _result(state, E_nuc, converged, ints, precision=None):
    return SCFResult(
        converged=converged,
        state=state,
        energy=float(state.energy) + float(E_nuc),
        E_elec=float(state.energy),
        E_nuc=float(E_nuc),
        n_iterations=state.iteration,
        S=ints.S,
        H_core=ints.H_core,
        ERI=ints.ERI,
        precision=precision,
    )


def run_rhf(mol, ints, config: Optional[CalcConfig] = None, timer: Optional[StageTimer] = None) -> SCFResult:
    """Closed-shell SCF to convergence (``rhf.py:95-169``)."""
    config = config or CalcConfig()
    if mol.spin != 0:
        raise ValueError(f"run_rhf requires a closed-shell molecule (spin=0); got spin={mol.spin}.")
    if mol.n_electrons % 2 != 0:
        raise ValueError(f"run_rhf requires an even number of electrons; got {mol.n_electrons}.")
    n_occ = mol.n_electrons // 2
    fb = FockBuilder(ints.ERI, config)
    dev = fb.device
    S = _t(ints.S, dev)
    H = _t(ints.H_core, dev)
    with optional_stage(timer, "scf", "monad"):
        with optional_stage(timer, "orthogonalize", "applicative"):
            X = symmetric_orthogonalization(S)
        with optional_stage(timer, "initial_guess", "applicative"):
            _, C = _diagonalize(H, X)
            D = 2.0 * C[:, :n_occ] @ C[:, :n_occ].T
            F = fb.rhf(H, D)
            eps, C = _diagonalize(F, X)
            E = float(0.5 * torch.sum(D * (H + F)))
        state = SCFState(density=D, fock=F, coefficients=C, orbital_energies=eps, energy=E, iteration=0)
        diis = DIIS(config.diis_space)
        converged = False
        last = E
        for _ in range(config.max_scf_iter):
            with optional_stage(timer, "fock_build", "applicative"):
                Fn = fb.rhf(H, state.density)
            with optional_stage(timer, "damp", "applicative"):
                if config.damping > 0.0:
                    Fn = (1.0 - config.damping) * Fn + config.damping * state.fock
            with optional_stage(timer, "diis", "applicative"):
                err = diis_error(Fn, state.density, S, X)
                Fx = diis.extrapolate(Fn, err)
            with optional_stage(timer, "diag", "applicative"):
                eps, C = _diagonalize(Fx, X)
            with optional_stage(timer, "density", "applicative"):
                D = 2.0 * C[:, :n_occ] @ C[:, :n_occ].T
            with optional_stage(timer, "energy", "foldable"):
                E = float(0.5 * torch.sum(D * (H + Fx)))
            state = SCFState(density=D, fock=Fx, coefficients=C, orbital_energies=eps, energy=E,
                             iteration=state.iteration + 1)
            dE = abs(E - last)
            err_max = float(torch.max(torch.abs(err)))
            last = E
            if fb.observe(err_max) and config.diis_reset_at_switch:
                diis.clear()  # the extrapolated F (and E) must not mix in the mixed-phase Fock matrices
            if dE < config.scf_conv and err_max < max(config.scf_conv, 1e-6) and fb.converged_ok():
                converged = True
                break
    return _result(state, ints.E_nuc, converged, ints, fb.record())


def run_uhf(mol, ints, config: Optional[CalcConfig] = None, timer: Optional[StageTimer] = None) -> SCFResult:
    """Open-shell SCF (``uhf.py:187-287``); result holds the total density."""
    config = config or CalcConfig(method="uhf")
    na, nb = mol.n_alpha, mol.n_beta
    fb = FockBuilder(ints.ERI, config)
    dev = fb.device
    S = _t(ints.S, dev)
    H = _t(ints.H_core, dev)
    n = S.shape[0]
    with optional_stage(timer, "scf", "monad"):
        with optional_stage(timer, "orthogonalize", "applicative"):
            X = symmetric_orthogonalization(S)
        with optional_stage(timer, "initial_guess", "applicative"):
            _, Ca = _diagonalize(H, X)
            if na != nb:
                Dai = Ca[:, :na] @ Ca[:, :na].T
                Ja, Ka = fb.jk(Dai)
                Fb_eff = H + Ja - Ka
                ev = torch.linalg.eigvalsh(X.T @ Fb_eff @ X)
                scale = 0.01 * float(ev.max() - ev.min()) + 0.1
                idx = torch.arange(n, dtype=torch.float64, device=dev)
                noise = scale * torch.outer(torch.sin(idx * 1.23 + 0.45), torch.cos(idx * 0.67 + 0.89))
                _, Cb = _diagonalize(Fb_eff + (noise + noise.T) / 2.0, X)
            else:
                Cb = Ca
            Da = Ca[:, :na] @ Ca[:, :na].T
            Db = Cb[:, :nb] @ Cb[:, :nb].T
            Fa, Fb = fb.uhf(H, Da, Db)
            ea, Ca = _diagonalize(Fa, X)
            eb, Cb = _diagonalize(Fb, X)
            Da = Ca[:, :na] @ Ca[:, :na].T
            Db = Cb[:, :nb] @ Cb[:, :nb].T
            E = float(0.5 * torch.sum(Da * (H + Fa)) + 0.5 * torch.sum(Db * (H + Fb)))
        diis = DIIS(config.diis_space)
        converged = False
        last = E
        it = 0
        init_damp = 0.3 if na != nb else 0.0
        for it in range(config.max_scf_iter):
            dmp = init_damp if it < 5 else config.damping
            with optional_stage(timer, "fock_build", "applicative"):
                Fan, Fbn = fb.uhf(H, Da, Db)
            with optional_stage(timer, "damp", "applicative"):
                if dmp > 0.0:
                    Fan = (1.0 - dmp) * Fan + dmp * Fa
                    Fbn = (1.0 - dmp) * Fbn + dmp * Fb
            with optional_stage(timer, "diis", "applicative"):
                e_a = diis_error(Fan, Da, S, X)
                e_b = diis_error(Fbn, Db, S, X)
                Fc = diis.extrapolate(torch.cat([Fan, Fbn]), torch.cat([e_a, e_b]))
                Fa, Fb = Fc[:n], Fc[n:]
            with optional_stage(timer, "diag", "applicative"):
                ea, Ca = _diagonalize(Fa, X)
                eb, Cb = _diagonalize(Fb, X)
            with optional_stage(timer, "density", "applicative"):
                Da = Ca[:, :na] @ Ca[:, :na].T
                Db = Cb[:, :nb] @ Cb[:, :nb].T
            with optional_stage(timer, "energy", "foldable"):
                E = float(0.5 * torch.sum(Da * (H + Fa)) + 0.5 * torch.sum(Db * (H + Fb)))
            err = max(float(torch.max(torch.abs(e_a))), float(torch.max(torch.abs(e_b))))
            dE = abs(E - last)
            last = E
            if fb.observe(err) and config.diis_reset_at_switch:
                diis.clear()
            if dE < config.scf_conv and err < max(config.scf_conv, 1e-6) and fb.converged_ok():
                converged = True
                break
    state = SCFState(density=Da + Db, fock=Fa, coefficients=Ca, orbital_energies=ea, energy=E, iteration=it + 1)
    res = _result(state, ints.E_nuc, converged, ints, fb.record())
    return res.replace(precision=dict(res.precision or {}, density_alpha=Da, density_beta=Db, fock_beta=Fb,
                                      coefficients_beta=Cb, orbital_energies_beta=eb))


def run_scf(mol, ints, config: Optional[CalcConfig] = None, timer: Optional[StageTimer] = None) -> SCFResult:
    """Dispatch on ``config.method`` (``scf/interface.py:17-31``)."""
    config = config or CalcConfig()
    m = config.method.lower()
    if m == "rhf":
        return run_rhf(mol, ints, config, timer)
    if m == "uhf":
        return run_uhf(mol, ints, config, timer)
    raise NotImplementedError(f"SCF method '{config.method}' is not implemented; available: rhf, uhf.")
