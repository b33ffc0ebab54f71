"""Integral entry points (``jax_qc/integrals/interface.py:26-67`` and
``jax_qc/integrals/eri.py:69-105``) on the device.

``compute_integrals`` returns an IntegralSet whose ERI field is a
:class:`DirectERI` handle: the SCF contracts against it with the fused
kernels, and the N^4 tensor is never built.  ``compute_eri_tensor`` is the
dense drop-in for small systems and parity checks.
"""

from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from .core import IntegralSet
from .engine import DirectERI
from .profiling import StageTimer, optional_stage


def nuclear_repulsion_energy(mol) -> float:
    """sum_{A<B} Z_A Z_B / R_AB (``nuclear.py:84-98``)."""
    xyz = np.asarray(mol.coords, dtype=np.float64)
    Z = np.asarray(mol.atomic_numbers, dtype=np.float64)
    total = 0.0
    for i in range(len(Z)):
        for j in range(i + 1, len(Z)):
            r = float(np.linalg.norm(xyz[i] - xyz[j]))
            if r == 0.0:
                raise ValueError(f"Atoms {i} and {j} are coincident; cannot compute E_nuc.")
            total += Z[i] * Z[j] / r
    return total


def compute_integrals(mol, basis, timer: Optional[StageTimer] = None, device=None,
                      schwarz_tau: float = 1e-13, engine: Optional[DirectERI] = None) -> IntegralSet:
    """S, T, V, H_core on the device and a DirectERI handle in place of the
    dense ERI tensor (same stage names as the reference)."""
    with optional_stage(timer, "integrals", "applicative"):
        with optional_stage(timer, "eri", "applicative"):
            eng = engine if engine is not None else DirectERI(basis, mol, device=device, schwarz_tau=schwarz_tau)
        with optional_stage(timer, "overlap", "applicative"):
            S, T, V = eng.one_electron()
        with optional_stage(timer, "h_core", "applicative"):
            H = T + V
        with optional_stage(timer, "nuclear_repulsion", "foldable"):
            E_nuc = nuclear_repulsion_energy(mol)
    return IntegralSet(S=S, T=T, V=V, H_core=H, ERI=eng, E_nuc=float(E_nuc))


def compute_eri_tensor(basis, device=None, max_bytes: int = 32 << 30):
    """Dense (n,n,n,n) ERI tensor (``eri.py:69-105``), exact (no screening)."""
    eng = DirectERI(basis, None, device=device, schwarz_tau=0.0)
    try:
        return eng.eri_tensor(max_bytes=max_bytes)
    finally:
        eng.close()
