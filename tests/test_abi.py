"""Host-side checks that need no GPU: the C ABI library loads and exports
every entry point include/jqc.h declares, signatures are bound, the basis
layer and flop model behave, and the product refuses to run without CUDA."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from jax_examples_b200 import _abi, flops
from jax_examples_b200 import basis as pb
from jax_examples_b200.core import cartesian_components, make_molecule


def test_library_exports_every_header_symbol(libjqc):
    declared = _abi.header_symbols()
    assert len(declared) >= 10
    for name in declared:
        assert hasattr(libjqc, name), name
        assert name in _abi.SIGNATURES, f"{name} has no ctypes signature"


def test_version_and_error_string(libjqc):
    assert libjqc.jqc_version() >= 100
    assert isinstance(libjqc.jqc_last_error(), bytes)


def test_invalid_arguments_rejected_before_any_gpu_work(libjqc):
    # mmax out of range and n < 0 are rejected on the host (no device call)
    with pytest.raises(ValueError):
        _abi.call("jqc_boys", None, 10, 99, None, 0, None)
    with pytest.raises(ValueError):
        _abi.call("jqc_boys", None, -1, 3, None, 0, None)
    with pytest.raises(NotImplementedError):
        _abi.call("jqc_eri_prim_quartets", 3, 0, 0, 0, 1, None, None, None, None)
    with pytest.raises(NotImplementedError):
        _abi.call("jqc_eri_prim_quartets", 0, 1, 0, 0, 1, None, None, None, None)
    with pytest.raises(ValueError):
        _abi.call("jqc_jk", None, 1, None, None, None, 0, 0.0, 0.0, None)


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback():
    from jax_examples_b200 import DirectERI

    mol = make_molecule(("H", "H"), [[0, 0, 0], [0, 0, 1.4]], [1, 1])
    with pytest.raises(RuntimeError, match="CUDA"):
        DirectERI(pb.build_basis_set(mol, "sto-3g"), mol)


def test_cartesian_order_is_libint():
    assert cartesian_components(1) == ((1, 0, 0), (0, 1, 0), (0, 0, 1))
    assert cartesian_components(2) == ((2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2))


def test_flop_model_frozen_values():
    assert flops.prim_quartet_flops(0, 0, 0, 0) == 34
    assert flops.prim_quartet_flops(1, 1, 1, 1) == 1434
    assert flops.prim_quartet_flops(2, 2, 2, 2) == 48754
    assert flops.prim_quartet_flops(2, 0, 1, 0) == 353


def test_water_cluster_shapes():
    for n, nbf, nbf2 in ((1, 19, 25), (8, 152, 200), (16, 304, 400)):
        mol = pb.water_cluster(n, seed=0)
        assert mol.n_electrons == 10 * n
        for prefix in ("", "syn-"):
            assert pb.build_basis_set(mol, prefix + "6-31g*").n_basis == nbf
            assert pb.build_basis_set(mol, prefix + "6-31g**").n_basis == nbf2
    # lattice spacing 2.9 A between O atoms
    mol = pb.water_cluster(8, seed=3)
    O = mol.coords[0::3]
    d = np.linalg.norm(O[1] - O[0]) * 0.529177210903
    assert abs(d - 2.9) < 1e-12


def test_published_basis_shapes():
    """Shell structure of the published bases for water: 18 spherical
    functions in 6-31G* (the reference's tests/test_basis.py:191-206), 7 in
    STO-3G; contraction lengths of 6-31G (O 1s has six primitives)."""
    mol = pb.water_cluster(1)
    assert pb.build_basis_set(mol, "6-31g*", spherical=True).n_basis == 18
    assert pb.build_basis_set(mol, "6-31g**", spherical=True).n_basis == 24
    bs = pb.build_basis_set(mol, "sto-3g")
    assert bs.n_basis == 7 and [s.angular_momentum for s in bs.shells] == [0, 0, 1, 0, 0]
    bs = pb.build_basis_set(mol, "6-31g*")
    o = [(s.angular_momentum, len(s.exponents)) for s in bs.shells if s.atom_index == 0]
    assert o == [(0, 6), (0, 3), (0, 1), (1, 3), (1, 1), (2, 1)]
    h = [(s.angular_momentum, len(s.exponents)) for s in pb.build_basis_set(mol, "6-31g**").shells if s.atom_index == 1]
    assert h == [(0, 3), (0, 1), (1, 1)]


def test_basis_errors_mirror_reference():
    mol = make_molecule(("Li",), [[0, 0, 0]], [3], spin=1)
    with pytest.raises(KeyError):
        pb.build_basis_set(mol, "syn-6-31g*")
    with pytest.raises(ValueError):
        make_molecule(("H",), [[0, 0, 0]], [1], spin=0)
