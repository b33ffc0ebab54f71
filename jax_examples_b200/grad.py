"""Analytic nuclear gradients on the device (replaces ``jax_qc/grad``).

The reference's "analytic" gradient (``grad/rhf_grad.py:106-211``) evaluates

    dE/dR = dE_nuc/dR + sum D dH/dR + 1/2 sum D (dJ - dK/2) - sum W dS/dR

with dH, dS and dERI from central finite differences of whole integral sets
(6 N_atoms full ERI builds).  Here the same expression is evaluated
analytically: the two-electron term by the ERI-derivative adjoint kernel
(``jqc_grad2e``: Gamma = D (x) D - exchange contracted with d(ab|cd)/dR on
the fly, never stored), the one-electron terms by ``jqc_grad1e``, and
dE_nuc/dR in closed form.

The pieces are exposed as ``torch.autograd.Function``s so a geometry
optimizer (or any torch code) can differentiate the SCF Lagrangian
    L(R) = E_nuc(R) + Tr[D H(R)] + 1/2 E2[D](R) - Tr[W S(R)]
with respect to the nuclear coordinates: at the converged D and W its
gradient is the SCF energy gradient.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _abi
from .engine import DirectERI, _ptr, _stream


def energy_weighted_density(C: torch.Tensor, eps: torch.Tensor, n_occ: int, occ: float = 2.0) -> torch.Tensor:
    """W = occ * sum_i^occ eps_i C_i C_i^T (``rhf_grad.py:92-103``)."""
    Co = C[:, :n_occ]
    return occ * (Co * eps[:n_occ][None, :]) @ Co.T


def nuclear_repulsion_gradient(coords, Z) -> torch.Tensor:
    """dE_nuc/dR_A = -sum_B Z_A Z_B (R_A - R_B) / |R_A - R_B|^3."""
    R = torch.as_tensor(np.asarray(coords), dtype=torch.float64)
    Zt = torch.as_tensor(np.asarray(Z), dtype=torch.float64)
    d = R[:, None, :] - R[None, :, :]
    r = torch.linalg.norm(d, dim=-1)
    r.fill_diagonal_(1.0)
    w = (Zt[:, None] * Zt[None, :]) / r ** 3
    w.fill_diagonal_(0.0)
    return -(w[:, :, None] * d).sum(dim=1)


def _cart(engine: DirectERI, M: torch.Tensor) -> torch.Tensor:
    return engine._to_cart(M).contiguous()


def grad_two_electron(engine: DirectERI, dens, j_scale: float, k_scale: float, dens_tau: float = 0.0,
                      class_ms: Optional[list] = None) -> torch.Tensor:
    """1/2 sum Gamma d(ab|cd)/dR, (n_atom, 3).  dens_tau > 0 skips quartets
    whose Gamma bound times Q_ab Q_cd is below it; a list passed as class_ms
    receives the 21 per-class kernel times (ms, classes serialised)."""
    D = torch.stack([_cart(engine, d) for d in dens]).contiguous()
    g = torch.zeros((len(engine.atom_Z), 3), dtype=torch.float64, device=engine.device)
    ms = (ctypes.c_double * 21)() if class_ms is not None else None
    with torch.cuda.device(engine.device):
        _abi.call("jqc_grad2e_ex", engine._ctx, D.shape[0], _ptr(D), float(j_scale), float(k_scale),
                  float(dens_tau), _ptr(g), _stream(engine.device), ms)
    if class_ms is not None:
        class_ms[:] = list(ms)
    return g


def grad_one_electron(engine: DirectERI, D: torch.Tensor, W: torch.Tensor) -> torch.Tensor:
    """sum D d(T+V)/dR - sum W dS/dR, (n_atom, 3)."""
    Dc, Wc = _cart(engine, D), _cart(engine, W)
    g = torch.zeros((len(engine.atom_Z), 3), dtype=torch.float64, device=engine.device)
    with torch.cuda.device(engine.device):
        _abi.call("jqc_grad1e", engine._ctx, _ptr(Dc), _ptr(Wc), _ptr(g), _stream(engine.device))
    return g


class TwoElectronEnergy(torch.autograd.Function):
    """E2 = 1/2 sum Gamma (ab|cd) at fixed densities, as a function of the
    nuclear coordinates.  Forward uses the fused J/K kernel
    (E2 = 1/2 sum_s Tr[D_s (j J(D^t) - k K(D_s))]); backward is the
    ERI-derivative adjoint kernel."""

    @staticmethod
    def forward(ctx, coords, engine: DirectERI, dens, j_scale: float, k_scale: float):
        D = torch.stack(list(dens))
        J, K = engine.jk(D)
        Jt = J.sum(dim=0)
        e2 = 0.0
        for s in range(D.shape[0]):
            e2 = e2 + 0.5 * torch.sum(D[s] * (j_scale * Jt - k_scale * K[s]))
        ctx.engine, ctx.dens, ctx.scales = engine, D, (j_scale, k_scale)
        return e2.reshape(())

    @staticmethod
    def backward(ctx, gout):
        g = grad_two_electron(ctx.engine, ctx.dens, *ctx.scales)
        return (gout * g).to(gout.device), None, None, None, None


class OneElectronLagrangian(torch.autograd.Function):
    """Tr[D H(R)] - Tr[W S(R)] at fixed D, W; backward = ``jqc_grad1e``."""

    @staticmethod
    def forward(ctx, coords, engine: DirectERI, D, W):
        S, T, V = engine.one_electron()
        ctx.engine, ctx.D, ctx.W = engine, D, W
        return (torch.sum(D * (T + V)) - torch.sum(W * S)).reshape(())

    @staticmethod
    def backward(ctx, gout):
        return (gout * grad_one_electron(ctx.engine, ctx.D, ctx.W)).to(gout.device), None, None, None


def _nuclear_repulsion_torch(coords, Z):
    n = coords.shape[0]
    i, j = torch.triu_indices(n, n, 1)
    r = torch.linalg.norm(coords[i] - coords[j], dim=-1)
    return torch.sum(Z[i] * Z[j] / r)


def scf_lagrangian(coords: torch.Tensor, Z, engine: DirectERI, D, W, dens, j_scale, k_scale):
    """L(R) whose gradient at the converged D, W is the SCF gradient."""
    Zt = torch.as_tensor(np.asarray(Z), dtype=torch.float64, device=coords.device)
    return (_nuclear_repulsion_torch(coords, Zt) + OneElectronLagrangian.apply(coords, engine, D, W)
            + TwoElectronEnergy.apply(coords, engine, dens, j_scale, k_scale))


def _engine_for(mol, result, basis, engine):
    if engine is not None:
        return engine
    if isinstance(getattr(result, "ERI", None), DirectERI):
        return result.ERI
    if basis is None:
        raise ValueError("need the basis (or an engine) of the converged calculation")
    return DirectERI(basis, mol)


def rhf_gradient(mol, result, basis=None, engine: Optional[DirectERI] = None, autograd: bool = False,
                 dens_tau: float = 0.0):
    """Analytic RHF gradient (n_atoms, 3) in Hartree/bohr; same expression as
    ``rhf_grad.py:106-211`` without finite differences.  dens_tau > 0 skips
    two-electron quartets whose density-weighted bound is below it (the
    mixed path's gradient; 0 = every Schwarz-surviving quartet)."""
    eng = _engine_for(mol, result, basis, engine)
    dev = eng.device
    st = result.state
    D = torch.as_tensor(st.density, dtype=torch.float64, device=dev)
    C = torch.as_tensor(st.coefficients, dtype=torch.float64, device=dev)
    eps = torch.as_tensor(st.orbital_energies, dtype=torch.float64, device=dev)
    W = energy_weighted_density(C, eps, mol.n_electrons // 2)
    if autograd:
        coords = torch.tensor(np.asarray(mol.coords), dtype=torch.float64, device=dev, requires_grad=True)
        L = scf_lagrangian(coords, mol.atomic_numbers, eng, D, W, [D], 1.0, 0.5)
        (g,) = torch.autograd.grad(L, coords)
        return g
    g = nuclear_repulsion_gradient(mol.coords, mol.atomic_numbers).to(dev)
    g = g + grad_one_electron(eng, D, W) + grad_two_electron(eng, [D], 1.0, 0.5, dens_tau)
    return g


def uhf_gradient(mol, result, basis=None, engine: Optional[DirectERI] = None):
    """Analytic UHF gradient: W = sum_s eps_si C_si C_si^T, Gamma with
    (D_alpha, D_beta), j = k = 1.  (The reference has no UHF analytic
    gradient; its numerical_gradient is the check.)"""
    eng = _engine_for(mol, result, basis, engine)
    dev = eng.device
    x = result.precision
    Da = torch.as_tensor(x["density_alpha"], dtype=torch.float64, device=dev)
    Db = torch.as_tensor(x["density_beta"], dtype=torch.float64, device=dev)
    Ca = torch.as_tensor(result.state.coefficients, dtype=torch.float64, device=dev)
    ea = torch.as_tensor(result.state.orbital_energies, dtype=torch.float64, device=dev)
    Cb = torch.as_tensor(x["coefficients_beta"], dtype=torch.float64, device=dev)
    eb = torch.as_tensor(x["orbital_energies_beta"], dtype=torch.float64, device=dev)
    W = energy_weighted_density(Ca, ea, mol.n_alpha, 1.0) + energy_weighted_density(Cb, eb, mol.n_beta, 1.0)
    g = nuclear_repulsion_gradient(mol.coords, mol.atomic_numbers).to(dev)
    g = g + grad_one_electron(eng, Da + Db, W) + grad_two_electron(eng, [Da, Db], 1.0, 1.0)
    return g


def compute_gradient(mol, result, basis=None, method: str = "analytic", engine=None, **kw):
    """Dispatcher (``grad/interface.py:20-55``): 'analytic' or 'numerical'."""
    if method == "analytic":
        if mol.spin == 0:
            return rhf_gradient(mol, result, basis=basis, engine=engine)
        return uhf_gradient(mol, result, basis=basis, engine=engine)
    if method == "numerical":
        return numerical_gradient(mol, basis_name=kw.get("basis_name"), step_size=kw.get("step_size", 1e-4))
    raise ValueError(f"Unknown gradient method '{method}'; expected 'analytic' or 'numerical'.")


def numerical_gradient(mol, basis_name, step_size: float = 1e-4, scf_conv: float = 1e-10, device=None):
    """Central finite differences of the total SCF energy
    (``grad/numerical_grad.py:51-94``), every energy on the device."""
    from .basis import build_basis_set
    from .core import CalcConfig, make_molecule
    from .integrals import compute_integrals
    from .scf import run_scf

    coords = np.asarray(mol.coords, dtype=np.float64)
    cfg = CalcConfig(method="rhf" if mol.spin == 0 else "uhf", scf_conv=scf_conv, max_scf_iter=200)
    g = np.zeros_like(coords)

    def energy(c):
        m = make_molecule(mol.elements, c, mol.atomic_numbers, mol.charge, mol.spin)
        ints = compute_integrals(m, build_basis_set(m, basis_name), device=device)
        return float(run_scf(m, ints, cfg).energy)

    for a in range(coords.shape[0]):
        for k in range(3):
            cp, cm = coords.copy(), coords.copy()
            cp[a, k] += step_size
            cm[a, k] -= step_size
            g[a, k] = (energy(cp) - energy(cm)) / (2 * step_size)
    return torch.as_tensor(g)
