"""Host-side data model of the two-electron path.

These mirror the reference's frozen data types (``jax_qc/core/types.py:40-201``)
field for field, so a caller holding a reference ``Shell``/``BasisSet``/
``Molecule`` can hand it straight to this package (every function here reads
attributes only, never ``isinstance``).  Arrays are NumPy on the host; device
copies live in :class:`jax_examples_b200.engine.DirectERI`.
"""

from __future__ import annotations

import dataclasses
from dataclasses import dataclass
from typing import Any, Optional, Tuple

import numpy as np

# CODATA 2018, as in jax_qc/core/constants.py:14-16.
BOHR_TO_ANGSTROM = 0.529177210903
ANGSTROM_TO_BOHR = 1.0 / BOHR_TO_ANGSTROM

ELEMENT_SYMBOLS = ("X", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne")
SYMBOL_TO_Z = {s: z for z, s in enumerate(ELEMENT_SYMBOLS)}


def symbol_to_z(symbol: str) -> int:
    key = symbol.strip().title()
    if key not in SYMBOL_TO_Z:
        raise ValueError(f"Unknown element symbol: {symbol!r}")
    return SYMBOL_TO_Z[key]


class _Replace:
    def replace(self, **changes):
        return dataclasses.replace(self, **changes)


@dataclass(frozen=True, eq=False)
class Shell(_Replace):
    """Contracted shell (``jax_qc/core/types.py:40-61``).

    ``coefficients`` already hold contraction coefficient x primitive norm x
    shell norm, exactly as the reference's ``normalize_shell`` returns them.
    """

    angular_momentum: int
    exponents: np.ndarray
    coefficients: np.ndarray
    center: np.ndarray
    atom_index: int


@dataclass(frozen=True, eq=False)
class BasisSet(_Replace):
    """Basis set (``jax_qc/core/types.py:64-85``)."""

    shells: tuple
    n_basis: int
    shell_to_basis: tuple
    basis_to_atom: np.ndarray
    name: str = ""
    spherical: bool = True


@dataclass(frozen=True, eq=False)
class Molecule(_Replace):
    """Molecule, coordinates in bohr (``jax_qc/core/types.py:88-109``)."""

    coords: np.ndarray
    atomic_numbers: np.ndarray
    elements: Tuple[str, ...]
    charge: int = 0
    spin: int = 0
    n_electrons: int = 0
    n_alpha: int = 0
    n_beta: int = 0


@dataclass(frozen=True, eq=False)
class IntegralSet(_Replace):
    """Integrals consumed by the SCF (``jax_qc/core/types.py:112-124``).

    ``ERI`` is either a dense (n,n,n,n) tensor or a
    :class:`~jax_examples_b200.engine.DirectERI` handle; the SCF drivers
    accept both, and with the handle the N^4 tensor never exists.
    """

    S: Any
    T: Any
    V: Any
    H_core: Any
    ERI: Any
    E_nuc: float


@dataclass(frozen=True, eq=False)
class SCFState(_Replace):
    """SCF iteration state (``jax_qc/core/types.py:127-138``)."""

    density: Any
    fock: Any
    coefficients: Any
    orbital_energies: Any
    energy: float
    iteration: int


@dataclass(frozen=True, eq=False)
class SCFResult(_Replace):
    """Converged SCF result (``jax_qc/core/types.py:141-150``)."""

    converged: bool
    state: SCFState
    energy: float
    E_elec: float
    E_nuc: float
    n_iterations: int
    S: Any
    H_core: Any
    ERI: Optional[Any] = None
    # Per-result accuracy record of the mixed-precision path (None for FP64).
    precision: Optional[dict] = None


@dataclass(frozen=True, eq=False)
class CalcConfig(_Replace):
    """Calculation configuration (``jax_qc/core/types.py:153-166``) plus the
    knobs of the direct two-electron engine.

    precision:      "fp64" (plain kernel) or "mixed" (FP32 for quartets whose
                    Schwarz bound is below ``mixed_tau``).
    schwarz_tau:    quartets with Q_ij*Q_kl*max|D| below this are skipped.
    mixed_tau:      FP32/FP64 split on the quartet Schwarz bound (1e-4: on
                    (H2O)16 the mixed builds are ~7% faster than at 1e-7 with
                    the same iterations and final error; 1e-2 and above cost
                    extra SCF iterations).
    fp64_switch:    max|DIIS error| below which the mixed policy switches to
                    FP64 (1e-4: 25-26 iterations on (H2O)16 instead of 28 at
                    1e-5, with the DIIS history cleared at the switch).
    fp64_tail_iters: in mixed mode, once the SCF is within ``fp64_switch`` of
                    convergence the remaining iterations use incremental FP64
                    builds; at least this many FP64 iterations are run.
    incremental:    build F from the density change dD when true.
    mixed_dens_tau: density-screening threshold of the incremental builds
                    in the mixed phase.
    mixed_dens_rel: those builds screen at max(mixed_dens_tau, mixed_dens_rel
                    x max|DIIS error| of the previous iteration) (1e-6: the
                    first iterations' Fock matrices only need the accuracy
                    of their SCF error; on (H2O)8-16 clusters 4-10% fewer Fock
                    seconds at the same errors; 1e-5 and above cost erratic
                    extra iterations).  Single-molecule builder only.
    fp64_tail_dens_tau: density-screening threshold of the incremental FP64
                    builds after the switch (mixed mode only; plain FP64
                    incremental builds screen at 1e-12).
    mixed_full_dens_tau: density-screening threshold of the full builds of
                    the mixed phase (their errors are dropped at the switch).
    fp64_switch_dens_tau: density-screening threshold of the full FP64 build
                    at the switch (mixed mode only; plain FP64 builds are
                    unscreened).
                    The five thresholds were swept together on (H2O)16 and
                    the 64-cluster sweep in 6-31G*, against FP64 converged
                    to 1e-10: these defaults give 80.3 ms of Fock builds on
                    (H2O)16 (88.4 ms with the previous 1e-5 / 1e-8 / 1e-11 /
                    1e-9 / 0) at 5.6e-8 Eh, and the sweep's largest error
                    1.9e-7 Eh (4.0e-8 before) in 0.67 s instead of 0.76 s.
    diis_reset_at_switch: clear the DIIS history when the mixed policy
                    switches to FP64, so the extrapolated Fock matrix of the
                    energy holds FP64 builds only.
    """

    method: str = "rhf"
    basis: str = "sto-3g"
    task: str = "energy"
    max_scf_iter: int = 128
    scf_conv: float = 1e-10
    diis_space: int = 8
    damping: float = 0.0
    guess: str = "core"
    verbose: int = 1
    profile: bool = False
    precision: str = "fp64"
    schwarz_tau: float = 1e-13
    mixed_tau: float = 1e-4
    fp64_tail_iters: int = 2
    fp64_switch: float = 1e-4
    incremental: bool = True
    mixed_dens_tau: float = 2e-8
    mixed_dens_rel: float = 1e-6
    fp64_tail_dens_tau: float = 1e-10
    mixed_full_dens_tau: float = 1e-8
    fp64_switch_dens_tau: float = 1e-11
    diis_reset_at_switch: bool = True


def make_molecule(elements, coords, atomic_numbers, charge: int = 0, spin: int = 0) -> Molecule:
    """Build a Molecule and derive electron counts (``jax_qc/core/types.py:169-201``).

    Raises ``ValueError`` on a negative electron count or a spin/parity
    mismatch, as the reference does.
    """
    Z = np.asarray(atomic_numbers, dtype=np.int64)
    n_electrons = int(Z.sum()) - int(charge)
    if n_electrons < 0:
        raise ValueError(
            f"Negative electron count: charge {charge} exceeds nuclear charge."
        )
    if (n_electrons - int(spin)) % 2 != 0:
        raise ValueError(
            f"Inconsistent spin: n_electrons={n_electrons}, 2S={spin} "
            "have different parity."
        )
    n_beta = (n_electrons - int(spin)) // 2
    n_alpha = n_electrons - n_beta
    return Molecule(
        coords=np.asarray(coords, dtype=np.float64),
        atomic_numbers=Z.astype(np.int32),
        elements=tuple(elements),
        charge=int(charge),
        spin=int(spin),
        n_electrons=n_electrons,
        n_alpha=n_alpha,
        n_beta=n_beta,
    )


def n_cartesian(l: int) -> int:
    """(l+1)(l+2)/2 Cartesian components (``mcmurchie_davidson.py:53-55``)."""
    return (l + 1) * (l + 2) // 2


def cartesian_components(l: int):
    """(lx, ly, lz) in libint order: lx descending, then ly descending
    (``mcmurchie_davidson.py:39-50``)."""
    out = []
    for lx in range(l, -1, -1):
        for ly in range(l - lx, -1, -1):
            out.append((lx, ly, l - lx - ly))
    return tuple(out)


def shell_offsets(shells, spherical: bool):
    """Cumulative basis-function offsets per shell (``overlap.py:58-64``)."""
    offsets = [0]
    for sh in shells:
        l = int(sh.angular_momentum)
        offsets.append(offsets[-1] + ((2 * l + 1) if spherical else n_cartesian(l)))
    return offsets
