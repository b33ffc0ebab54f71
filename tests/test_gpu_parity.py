"""Parity of the sm_100a kernels (through the C ABI) with the oracle and the
reference's golden fixtures.  Tolerances are the ones the target states:
ERIs 1e-10 absolute, energies 1e-8 Eh (plain FP64 path)."""

from __future__ import annotations

import os

import numpy as np
import pytest
import torch

import oracle
from jax_examples_b200 import CalcConfig, DirectERI, boys, compute_integrals, eri_prim_quartets, run_scf
from jax_examples_b200 import basis as pb
from jax_examples_b200.core import make_molecule

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def test_boys_fp64_fp32_vs_quadrature():
    b = np.load(os.path.join(GOLDEN, "boys.npz"))
    T = torch.tensor(b["T"], device=DEV)
    true = b["true"]
    out = boys(T, true.shape[1] - 1).cpu().numpy()
    np.testing.assert_allclose(out, true, rtol=2e-14, atol=1e-300)
    out32 = boys(T, true.shape[1] - 1, fp32=True).cpu().numpy().astype(np.float64)
    np.testing.assert_allclose(out32, true, rtol=2e-6, atol=1e-37)


def test_boys_sweep_distribution_vs_oracle():
    """The Boys sweep distribution (half U[0,30], half log-U[1e-8,1e3]), m=0..8."""
    rng = np.random.default_rng(7)
    n = 1 << 16
    T = np.concatenate([rng.uniform(0, 30, n // 2), 10 ** rng.uniform(-8, 3, n // 2)])
    ref = oracle.boys_array(T, 8, mode=1)
    got = boys(torch.tensor(T, device=DEV), 8).cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=2e-14, atol=1e-300)


def _random_prim_quartets(cls, n, rng):
    ex = 10 ** rng.uniform(-1, 2, (n, 4))
    ctr = rng.uniform(0, 4.0 / 0.529177210903, (n, 4, 3))
    return ex, ctr


@pytest.mark.parametrize("cls", [(0, 0, 0, 0), (1, 0, 0, 0), (1, 1, 1, 1), (2, 0, 1, 0), (2, 2, 2, 2), (2, 1, 1, 0),
                                 (2, 2, 1, 1), (2, 1, 2, 1), (2, 2, 0, 0), (2, 1, 1, 1)])
def test_primitive_blocks_vs_oracle(cls):
    rng = np.random.default_rng(sum(cls) * 31 + cls[0])
    n = 64
    ex, ctr = _random_prim_quartets(cls, n, rng)
    got = eri_prim_quartets(cls, torch.tensor(ex, device=DEV), torch.tensor(ctr, device=DEV)).cpu().numpy()
    for q in range(n):
        ref = oracle.primitive_eri(ex[q, 0], ctr[q, 0], cls[0], ex[q, 1], ctr[q, 1], cls[1],
                                   ex[q, 2], ctr[q, 2], cls[2], ex[q, 3], ctr[q, 3], cls[3], mode=1)
        np.testing.assert_allclose(got[q], ref, rtol=0, atol=1e-10 * max(1.0, np.abs(ref).max()))


def test_primitive_blocks_vs_golden():
    m = np.load(os.path.join(GOLDEN, "mmd_primitives.npz"), allow_pickle=True)
    for c, acc in zip(m["pe_cases"], m["pe_acc"]):
        cls = tuple(int(x) for x in c[:4])
        ex = np.asarray(c[4:8])[None]
        ctr = np.asarray(c[8:]).reshape(1, 4, 3)
        # the kernels take canonical classes: swap pairs where needed
        la, lb, lc, ld = cls
        perm = [0, 1, 2, 3]
        if la < lb:
            perm[0], perm[1] = 1, 0
        if lc < ld:
            perm[2], perm[3] = 3, 2
        ref = np.asarray(acc, dtype=float).reshape([(l + 1) * (l + 2) // 2 for l in cls])
        ref = ref.transpose(perm)
        kcls = tuple(cls[p] for p in perm)
        pb_, pk_ = (kcls[0] * (kcls[0] + 1) // 2 + kcls[1]), (kcls[2] * (kcls[2] + 1) // 2 + kcls[3])
        if pb_ < pk_:
            perm2 = [2, 3, 0, 1]
            ref = ref.transpose(perm2)
            kcls = tuple(kcls[p] for p in perm2)
            perm = [perm[p] for p in perm2]
        got = eri_prim_quartets(kcls, torch.tensor(ex[:, perm], device=DEV),
                                torch.tensor(ctr[:, perm], device=DEV)).cpu().numpy()[0]
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-10 * max(1.0, np.abs(ref).max()))


@pytest.mark.parametrize("tag", ["water_synsto3g", "water_sto3g"])
def test_eri_tensor_water_sto3g_vs_golden(golden, tag):
    """Full 7^4 tensor of the STO-3G water (the reference's config-1 oracle
    case) against the reference's own tensor, and its 8-fold symmetry."""
    g = golden(tag)
    eng = DirectERI(g.basis(), g.molecule(), device=0, schwarz_tau=0.0)
    eri = eng.eri_tensor().cpu().numpy()
    np.testing.assert_allclose(eri, g.arr["eri"], atol=1e-10, rtol=0)
    # 8-fold symmetry
    np.testing.assert_allclose(eri, eri.transpose(1, 0, 2, 3), atol=0)
    np.testing.assert_allclose(eri, eri.transpose(2, 3, 0, 1), atol=0)


@pytest.mark.parametrize("tag", ["water_syn631gs", "water_631gs"])
def test_eri_tensor_water_631gs_vs_golden(golden, tag):
    g = golden(tag)
    eng = DirectERI(g.basis(), g.molecule(), device=0, schwarz_tau=0.0)
    eri = eng.eri_tensor().cpu().numpy()
    i = g.arr["eri_idx"]
    np.testing.assert_allclose(eri[i[:, 0], i[:, 1], i[:, 2], i[:, 3]], g.arr["eri_val"], atol=1e-10, rtol=0)
    ref = oracle.eri_tensor(g.basis(), mode=1)
    np.testing.assert_allclose(eri, ref, atol=1e-10, rtol=0)


REAL_AND_SYN = ["water_synsto3g", "water_syn631gs", "water_sto3g", "water_631gs", "water_631gss_sph"]


@pytest.mark.parametrize("tag", REAL_AND_SYN)
def test_one_electron_and_schwarz_vs_golden(golden, tag):
    g = golden(tag)
    eng = DirectERI(g.basis(), g.molecule(), device=0, schwarz_tau=0.0)
    S, T, V = (x.cpu().numpy() for x in eng.one_electron())
    np.testing.assert_allclose(S, g.arr["S"], atol=1e-12)
    np.testing.assert_allclose(T, g.arr["T"], atol=1e-12)
    np.testing.assert_allclose(V, g.arr["V"], atol=1e-11)
    np.testing.assert_allclose(eng.schwarz().cpu().numpy(), g.arr["Q"], atol=1e-12)


@pytest.mark.parametrize("tag", REAL_AND_SYN)
def test_jk_rhf_uhf_vs_golden(golden, tag):
    g = golden(tag)
    eng = DirectERI(g.basis(), g.molecule(), device=0, schwarz_tau=0.0)
    D = torch.tensor(g.arr["D_rand"], device=DEV)
    J, K = eng.jk(D)
    np.testing.assert_allclose((J - 0.5 * K).cpu().numpy(), g.arr["F_rand"], atol=1e-10)
    Db = torch.tensor(g.arr["D_rand_b"], device=DEV)
    J2, K2 = eng.jk(torch.stack([D, Db]))
    Jt = J2[0] + J2[1]
    np.testing.assert_allclose((Jt - K2[0]).cpu().numpy(), g.arr["Fa_rand"], atol=1e-10)
    np.testing.assert_allclose((Jt - K2[1]).cpu().numpy(), g.arr["Fb_rand"], atol=1e-10)


def test_jk_cluster_vs_oracle_direct():
    mol = pb.water_cluster(3, seed=1)
    bs = pb.build_basis_set(mol, "6-31g*")
    rng = np.random.default_rng(3)
    n = bs.n_basis
    D = rng.standard_normal((n, n)) * 0.05
    D = D + D.T
    Jr, Kr = oracle.jk_quartets(bs, D, mode=1)
    eng = DirectERI(bs, mol, device=0, schwarz_tau=0.0)
    J, K = eng.jk(torch.tensor(D, device=DEV))
    np.testing.assert_allclose(J.cpu().numpy(), Jr, atol=1e-10)
    np.testing.assert_allclose(K.cpu().numpy(), Kr, atol=1e-10)
    # screened (tau=1e-13) build stays within 1e-10 of the exact one
    eng2 = DirectERI(bs, mol, device=0, schwarz_tau=1e-13)
    J2, K2 = eng2.jk(torch.tensor(D, device=DEV))
    np.testing.assert_allclose(J2.cpu().numpy(), Jr, atol=1e-10)
    np.testing.assert_allclose(K2.cpu().numpy(), Kr, atol=1e-10)
    # mixed precision: bounded error, FP32 part non-empty
    st = eng2.stats("mixed", 1e-7)
    assert st["quartets_fp32"] > 0
    J3, K3 = eng2.jk(torch.tensor(D, device=DEV), precision="mixed", mixed_tau=1e-7)
    assert np.max(np.abs(J3.cpu().numpy() - Jr)) < 1e-7
    assert np.max(np.abs(K3.cpu().numpy() - Kr)) < 1e-7


def _screen_keep(pk, Q, D, tau=None):
    """The density-screening rule of the J/K kernels, restated in NumPy: a
    canonical quartet (ij|kl) is kept unless float(Q_ij) float(Q_kl) m < tau
    in FP32, m = max(2 d_ij, 2 d_kl, d_ik, d_il, d_jk, d_jl) over the FP32
    block maxima d of |D|.  Without tau, picks one in the middle of the
    widest relative gap between the bounds of the middle half of the quartets
    (so no bound sits within 0.1% of it) and returns it too."""
    off = pk.offsets
    ns = pk.n_shell
    dm = np.zeros((ns, ns), dtype=np.float32)
    for a in range(ns):
        for b in range(ns):
            dm[a, b] = np.float32(np.abs(D[off[a]:off[a + 1], off[b]:off[b + 1]]).max())
    qs = oracle.canonical_quartets(ns)
    i, j, k, l = qs.T
    two = np.float32(2.0)
    m = np.maximum.reduce([two * dm[i, j], two * dm[k, l], dm[i, k], dm[i, l], dm[j, k], dm[j, l]])
    Qf = Q.astype(np.float32)
    x = (Qf[i, j] * Qf[k, l]) * m
    if tau is None:
        v = np.unique(x[x > 0])
        lo, hi = len(v) // 4, 3 * len(v) // 4
        r = v[lo + 1:hi] / v[lo:hi - 1]
        g = int(np.argmax(r)) + lo
        assert v[g + 1] / v[g] > 1.001
        tau = float(np.sqrt(float(v[g]) * float(v[g + 1])))
    keep = ~(x < np.float32(tau))
    return qs, keep, tau


def test_density_screened_jk_vs_oracle_same_rule():
    """Density screening (block maxima, the bound against their largest, and
    the device-side compaction of work items that all fail it) drops exactly
    the quartets the rule drops: the oracle digesting the quartets the rule
    keeps matches the screened build at 1e-10, with a threshold that drops
    about half of them."""
    mol = pb.water_cluster(3, seed=1)
    bs = pb.build_basis_set(mol, "6-31g*")
    pk = oracle.Packed(bs)
    rng = np.random.default_rng(11)
    n = bs.n_basis
    # density blocks spanning many orders of magnitude: decay with the
    # distance between the functions' centres
    ctr = np.repeat(pk.centres, np.diff(pk.offsets), axis=0)
    r2 = ((ctr[:, None, :] - ctr[None, :, :]) ** 2).sum(-1)
    D = rng.standard_normal((n, n)) * np.exp(-0.3 * r2)
    D = D + D.T
    Q = oracle.schwarz(bs)
    qs, keep, tau = _screen_keep(pk, Q, D)
    assert 0.2 < keep.mean() < 0.8
    Jr, Kr = oracle.jk_quartets(bs, D, qs[keep])
    eng = DirectERI(bs, mol, device=0, schwarz_tau=0.0)
    for _ in range(2):  # the second build reuses the work list and its item bounds
        J, K = eng.jk(torch.tensor(D, device=DEV), dens_tau=tau)
        np.testing.assert_allclose(J.cpu().numpy(), Jr, atol=1e-10)
        np.testing.assert_allclose(K.cpu().numpy(), Kr, atol=1e-10)
    # a density below every bound: nothing survives the compaction
    J0, K0 = eng.jk(torch.tensor(D * 1e-30, device=DEV), dens_tau=tau)
    assert float(J0.abs().max()) == 0.0 and float(K0.abs().max()) == 0.0


def test_eri_tensor_spherical_vs_golden(golden):
    """6-31G** water in the solid-harmonic basis (the reference default):
    the tensor through the engine's spherical map against the reference's
    ``_spherical_eri_block`` values (``eri.py:61-66,100-103``)."""
    g = golden("water_631gss_sph")
    eng = DirectERI(g.basis(), g.molecule(), device=0, schwarz_tau=0.0)
    eri = eng.eri_tensor().cpu().numpy()
    assert eri.shape == (24,) * 4
    i = g.arr["eri_idx"]
    np.testing.assert_allclose(eri[i[:, 0], i[:, 1], i[:, 2], i[:, 3]], g.arr["eri_val"], atol=1e-10, rtol=0)


@pytest.mark.parametrize("tag", ["water_synsto3g", "water_syn631gs", "water_cation_synsto3g_uhf",
                                 "water_sto3g", "water_cation_sto3g_uhf", "water_631gs", "water_631gss_sph"])
def test_scf_energy_vs_golden(golden, tag):
    g = golden(tag)
    mol, bs = g.molecule(), g.basis()
    ints = compute_integrals(mol, bs, device=0, schwarz_tau=0.0)
    res = run_scf(mol, ints, CalcConfig(method="uhf" if mol.spin else "rhf", scf_conv=1e-10))
    assert res.converged
    assert abs(res.energy - g.rec["energy"]) < 1e-8


def test_tier1_golden_energies_gpu():
    import json

    data = json.load(open(os.path.join(GOLDEN, "tier1_sto3g.json")))
    for name, d in data.items():
        mol = make_molecule(tuple(d["elements"]), np.array(d["coords"], dtype=float), np.array(d["Z"]), d["charge"])
        ints = compute_integrals(mol, pb.build_basis_set(mol, "sto-3g"), device=0, schwarz_tau=0.0)
        res = run_scf(mol, ints, CalcConfig(scf_conv=1e-10))
        assert abs(res.energy - d["reference_energy"]) < 1e-8, name
        assert abs(res.energy - d["golden_pyscf"]) < 1e-6, name


def test_tier2_pyscf_energies_gpu():
    """examples/08_rhf_tier2.py:33-41 through the CUDA path in the spherical
    basis: the reference's own energies to 1e-8 Eh and, for water in STO-3G,
    6-31G and 6-31G**, the PySCF energies to 1e-8 Eh."""
    import json

    data = json.load(open(os.path.join(GOLDEN, "tier2_pyscf.json")))
    for key, d in data.items():
        mol = make_molecule(tuple(d["elements"]), np.array(d["coords"], dtype=float), np.array(d["Z"]))
        bs = pb.build_basis_set(mol, d["basis"], spherical=True)
        assert bs.n_basis == d["n_basis"]
        ints = compute_integrals(mol, bs, device=0, schwarz_tau=0.0)
        res = run_scf(mol, ints, CalcConfig(scf_conv=1e-10))
        assert res.converged, key
        assert abs(res.energy - d["reference_energy"]) < 1e-8, key
        if key.startswith("H2O/"):
            assert abs(res.energy - d["golden_pyscf"]) < 1e-8, key
