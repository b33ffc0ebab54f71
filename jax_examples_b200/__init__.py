"""jax_examples_b200: B200-native (sm_100a) two-electron engine behind the
jax_qc drop-in: McMurchie-Davidson ERIs over Schwarz-screened shell quartets
fused with J/K digestion, the ERI-derivative adjoint for nuclear gradients,
and the FP64 SCF drivers around them.  CUDA kernels live in libjqc.so
(``csrc/``, C ABI in ``include/jqc.h``); there is no CPU fallback."""

from .basis import build_basis_set, register_basis, water_cluster, water_monomer_bohr
from .core import (
    BasisSet,
    CalcConfig,
    IntegralSet,
    Molecule,
    SCFResult,
    SCFState,
    Shell,
    make_molecule,
)
from .engine import DirectERI, boys, eri_prim_quartets
from .fock import build_fock_rhf, build_fock_uhf
from .grad import compute_gradient, numerical_gradient, rhf_gradient, uhf_gradient
from .integrals import compute_eri_tensor, compute_integrals, nuclear_repulsion_energy
from .profiling import StageTimer
from .scf import run_rhf, run_scf, run_uhf

__all__ = [
    "BasisSet", "CalcConfig", "DirectERI", "IntegralSet", "Molecule", "SCFResult", "SCFState", "Shell",
    "StageTimer", "boys", "compute_gradient", "numerical_gradient", "rhf_gradient", "uhf_gradient", "build_basis_set", "build_fock_rhf", "build_fock_uhf", "compute_eri_tensor",
    "compute_integrals", "eri_prim_quartets", "make_molecule", "nuclear_repulsion_energy", "register_basis",
    "run_rhf", "run_scf", "run_uhf", "water_cluster", "water_monomer_bohr",
]
