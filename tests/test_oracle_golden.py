"""The CPU oracle (oracle/) against the reference's own outputs (golden
fixtures): this pins the oracle before it is used to check the CUDA path."""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

import oracle
from jax_examples_b200 import basis as pb
from jax_examples_b200.core import make_molecule

from conftest import GOLDEN


def test_boys_exact_matches_quadrature():
    b = np.load(os.path.join(GOLDEN, "boys.npz"))
    mine = np.array([[oracle.boys_exact(n, t) for n in range(b["true"].shape[1])] for t in b["T"]])
    np.testing.assert_allclose(mine, b["true"], rtol=1e-14, atol=0)


def test_boys_reference_restatement():
    """oracle.boys_ref restates boys.py:86-109 including its inaccuracy: equal to
    the reference where the reference is well conditioned, and just as wrong
    (order of magnitude) where the upward recurrence breaks down."""
    b = np.load(os.path.join(GOLDEN, "boys.npz"))
    T, ref, true = b["T"], b["ref"], b["true"]
    mine = np.array([[oracle.boys_ref(n, t) for n in range(ref.shape[1])] for t in T])
    good = np.abs(ref - true) < 1e-8 * np.abs(true)
    np.testing.assert_allclose(mine[good], ref[good], rtol=1e-7)
    bad = ~good
    assert bad.sum() > 0  # the reference's high-n / small-T breakdown is present
    np.testing.assert_array_equal(np.abs(mine[bad] - true[bad]) > 1e-9 * np.abs(true[bad]), True)


def test_hermite_e_exact():
    m = np.load(os.path.join(GOLDEN, "mmd_primitives.npz"), allow_pickle=True)
    for c, o in zip(m["he_cases"], m["he_out"]):
        la, lb = int(c[0]), int(c[1])
        np.testing.assert_allclose(oracle.hermite_e(la, lb, c[2], c[3], c[4]).ravel(), o, rtol=0, atol=1e-15)


def test_primitive_eri_both_boys():
    m = np.load(os.path.join(GOLDEN, "mmd_primitives.npz"), allow_pickle=True)
    for c, r0, r1 in zip(m["pe_cases"], m["pe_ref"], m["pe_acc"]):
        cls = [int(x) for x in c[:4]]
        ex = c[4:8]
        ctr = c[8:].reshape(4, 3)
        args = []
        for k in range(4):
            args += [ex[k], ctr[k], cls[k]]
        scale = max(1e-300, float(np.max(np.abs(r1))))
        np.testing.assert_allclose(oracle.primitive_eri(*args, mode=0).ravel(), r0, rtol=0, atol=1e-12 * max(scale, 1))
        np.testing.assert_allclose(oracle.primitive_eri(*args, mode=1).ravel(), r1, rtol=0, atol=1e-12 * max(scale, 1))


MOLECULE_TAGS = ["water_synsto3g", "water_syn631gs", "water_cation_synsto3g_uhf",
                 "water_sto3g", "water_cation_sto3g_uhf", "water_631gs", "water_631gss_sph"]


@pytest.mark.parametrize("tag", MOLECULE_TAGS)
def test_molecule_integrals_and_energy(golden, tag):
    g = golden(tag)
    mol, bs = g.molecule(), g.basis()
    a = g.arr
    # the package's basis layer reproduces the reference's normalized shells
    for s, c, l in zip(bs.shells, g.rec["shells"]["coefs"], g.rec["shells"]["l"]):
        assert s.angular_momentum == l
        np.testing.assert_allclose(s.coefficients, c, rtol=1e-15, atol=0)
    if bs.spherical:
        return _spherical_system(g, mol, bs)
    S, T, V = oracle.one_electron(bs, mol, mode=0)
    np.testing.assert_allclose(S, a["S"], atol=1e-13)
    np.testing.assert_allclose(T, a["T"], atol=1e-13)
    np.testing.assert_allclose(V, a["V"], atol=1e-12)
    np.testing.assert_allclose(oracle.schwarz(bs, mode=0), a["Q"], atol=1e-13)
    eri = oracle.eri_tensor(bs, mode=0)
    if "eri" in a:
        np.testing.assert_allclose(eri, a["eri"], atol=1e-13)
    if "eri_idx" in a:
        i = a["eri_idx"]
        np.testing.assert_allclose(eri[i[:, 0], i[:, 1], i[:, 2], i[:, 3]], a["eri_val"], atol=1e-12)
    J, K = oracle.jk_from_tensor(a["D_rand"], eri)
    np.testing.assert_allclose(J - 0.5 * K, a["F_rand"], atol=1e-12)
    Jd, Kd = oracle.jk_quartets(bs, a["D_rand"], mode=0)  # direct digestion == einsum on the tensor
    np.testing.assert_allclose(Jd, J, atol=1e-13)
    np.testing.assert_allclose(Kd, K, atol=1e-13)
    H = T + V
    enuc = oracle.nuclear_repulsion(mol.coords, mol.atomic_numbers)
    if mol.spin == 0:
        E = oracle.rhf(S, H, lambda D: oracle.jk_from_tensor(D, eri), mol.n_electrons // 2)[0]
    else:
        E = oracle.uhf(S, H, lambda D: oracle.jk_from_tensor(D, eri), mol.n_alpha, mol.n_beta)[0]
    assert abs(E + enuc - g.rec["energy"]) < 1e-10


def _spherical_system(g, mol, bs):
    """Spherical fixture (the reference default, ``basis/build.py:28``): the
    oracle's Cartesian integrals through the solid-harmonic map equal the
    reference's spherical ones (``eri.py:61-66,100-103``)."""
    a = g.arr
    C = oracle.spherical_matrix(bs)
    S, T, V = (C @ M @ C.T for M in oracle.one_electron(bs, mol, mode=0))
    np.testing.assert_allclose(S, a["S"], atol=1e-13)
    np.testing.assert_allclose(T, a["T"], atol=1e-13)
    np.testing.assert_allclose(V, a["V"], atol=1e-12)
    np.testing.assert_allclose(oracle.schwarz(bs, mode=0), a["Q"], atol=1e-13)
    eri_c = oracle.eri_tensor(bs, mode=0)
    eri = oracle.eri_to_spherical(eri_c, C)
    i = a["eri_idx"]
    np.testing.assert_allclose(eri[i[:, 0], i[:, 1], i[:, 2], i[:, 3]], a["eri_val"], atol=1e-12)
    J, K = oracle.jk_from_tensor(a["D_rand"], eri)
    np.testing.assert_allclose(J - 0.5 * K, a["F_rand"], atol=1e-12)
    Jc, Kc = oracle.jk_quartets(bs, C.T @ a["D_rand"] @ C, mode=0)  # direct digestion in the Cartesian layout
    np.testing.assert_allclose(C @ Jc @ C.T, J, atol=1e-12)
    np.testing.assert_allclose(C @ Kc @ C.T, K, atol=1e-12)
    E = oracle.rhf(S, T + V, lambda D: oracle.jk_from_tensor(D, eri), mol.n_electrons // 2)[0]
    assert abs(E + oracle.nuclear_repulsion(mol.coords, mol.atomic_numbers) - g.rec["energy"]) < 1e-10


@pytest.mark.parametrize("tag", ["water_synsto3g", "water_sto3g"])
def test_gradient_fd_restatement(golden, tag):
    g = golden(tag)
    mol = g.molecule()
    build = lambda m: pb.build_basis_set(m, g.rec["basis"])  # noqa: E731
    E, D, C, eps, ok = oracle.rhf_energy(mol, build, mode=0)
    grad = oracle.rhf_gradient_fd(mol, build, D, C, eps, mode=0,
                                  displace=lambda m, c: make_molecule(m.elements, c, m.atomic_numbers, m.charge, m.spin))
    np.testing.assert_allclose(grad, g.arr["grad"], atol=1e-9)


def test_tier1_golden_energies():
    """examples/07_rhf_scf.py:31-36 (PySCF STO-3G energies) reproduced by the
    oracle with the package's basis layer, to the reference test tolerance."""
    data = json.load(open(os.path.join(GOLDEN, "tier1_sto3g.json")))
    for name, d in data.items():
        mol = make_molecule(tuple(d["elements"]), np.array(d["coords"], dtype=float), np.array(d["Z"]), d["charge"])
        E = oracle.rhf_energy(mol, lambda m: pb.build_basis_set(m, "sto-3g"), mode=0)[0]
        assert abs(E - d["reference_energy"]) < 1e-9, name
        assert abs(E - d["golden_pyscf"]) < 1e-6, name


# The example's PySCF numbers for HF, CH4 and NH3 are not reproduced by the
# reference's own code on the published STO-3G tables either (it lands
# 1.1e-4, 2.3e-5 and 2.8e-2 Eh away); only the reference energy pins those.
PYSCF_PINNED = ("H2O/sto-3g", "H2O/6-31g", "H2O/6-31g**")


def test_tier2_pyscf_energies():
    """examples/08_rhf_tier2.py:33-41: the published bases (spherical, the
    reference default) through the oracle reproduce the reference's own RHF
    energies to 1e-9 Eh and, for water in STO-3G / 6-31G / 6-31G**, the PySCF
    energies to 1e-8 Eh (the example's own tolerance is 1e-6)."""
    data = json.load(open(os.path.join(GOLDEN, "tier2_pyscf.json")))
    assert set(PYSCF_PINNED) <= set(data)
    for key, d in data.items():
        mol = make_molecule(tuple(d["elements"]), np.array(d["coords"], dtype=float), np.array(d["Z"]))
        E = oracle.rhf_energy(mol, lambda m: pb.build_basis_set(m, d["basis"]), mode=0, spherical=True)[0]
        assert abs(E - d["reference_energy"]) < 1e-9, key
        if key in PYSCF_PINNED:
            assert abs(E - d["golden_pyscf"]) < 1e-8, key
