"""Batched path on the GPU: one context over molecules of uneven size
(jqc_batch_partition), CUDA-graph replay, per-class tuning and the autotuner,
lock-step RHF, batched gradients and the batched BFGS.  Every batched result
is checked against the same molecule run alone (itself pinned to the oracle
in test_gpu_parity / test_gpu_gradient) and, for one small batch, against the
oracle directly.  Tolerances: J/K 1e-10, energies 1e-8 Eh, gradients
1e-7 Eh/bohr (the plain FP64 path's)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from jax_examples_b200 import CalcConfig, DirectERI, _abi, compute_integrals, run_scf
from jax_examples_b200 import basis as pb
from jax_examples_b200.batch import (BATCH_DENS_TAU, BatchedERI, MoleculeBatch, optimize_bfgs_batch,
                                     rhf_gradient_batch, run_rhf_batch)
from jax_examples_b200.grad import rhf_gradient

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
BASIS = "6-31g*"


def _mols(sizes, seed=0, noise=0.05):
    return [pb.water_cluster(n, seed=seed + i, noise_angstrom=noise) for i, n in enumerate(sizes)]


def _random_block_density(batch, rng, scale=0.05):
    n = batch.n_basis
    D = np.zeros((n, n))
    for m in range(len(batch)):
        o, k = batch.bf_off[m], batch.n_bf[m]
        a = rng.standard_normal((k, k)) * scale
        D[o:o + k, o:o + k] = a + a.T
    return D


def test_batch_jk_matches_each_molecule_alone():
    batch = MoleculeBatch(_mols([1, 3, 2]), BASIS)
    eng = BatchedERI(batch, schwarz_tau=1e-12)
    rng = np.random.default_rng(3)
    D = torch.tensor(_random_block_density(batch, rng), device=DEV)[None].contiguous()
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    eng.jk_into(D, J, K)
    torch.cuda.synchronize()
    Jn, Kn = J[0].cpu().numpy(), K[0].cpu().numpy()
    mask = np.zeros_like(Jn, dtype=bool)
    for m, mol in enumerate(batch.mols):
        o, k = batch.bf_off[m], batch.n_bf[m]
        mask[o:o + k, o:o + k] = True
        single = DirectERI(batch.bases[m], mol, device=0, schwarz_tau=1e-12)
        Js, Ks = single.jk(D[0, o:o + k, o:o + k].contiguous())
        np.testing.assert_allclose(Jn[o:o + k, o:o + k], Js.cpu().numpy(), atol=1e-10, rtol=0)
        np.testing.assert_allclose(Kn[o:o + k, o:o + k], Ks.cpu().numpy(), atol=1e-10, rtol=0)
        single.close()
    assert np.all(Jn[~mask] == 0.0) and np.all(Kn[~mask] == 0.0)
    eng.close()


def test_batch_jk_vs_oracle_small():
    mols = [pb.water_cluster(1, seed=1, noise_angstrom=0.05), pb.water_cluster(1, seed=2, noise_angstrom=0.05)]
    batch = MoleculeBatch(mols, "sto-3g")
    eng = BatchedERI(batch, schwarz_tau=0.0)
    rng = np.random.default_rng(5)
    Dn = _random_block_density(batch, rng)
    D = torch.tensor(Dn, device=DEV)[None].contiguous()
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    eng.jk_into(D, J, K)
    for m in range(2):
        o, k = batch.bf_off[m], batch.n_bf[m]
        eri = oracle.eri_tensor(batch.bases[m])
        Jr, Kr = oracle.jk_from_tensor(np.ascontiguousarray(Dn[o:o + k, o:o + k]), eri)
        np.testing.assert_allclose(J[0, o:o + k, o:o + k].cpu().numpy(), Jr, atol=1e-10, rtol=0)
        np.testing.assert_allclose(K[0, o:o + k, o:o + k].cpu().numpy(), Kr, atol=1e-10, rtol=0)
    eng.close()


def test_batch_one_electron_matches_each_molecule():
    batch = MoleculeBatch(_mols([2, 1]), BASIS)
    eng = BatchedERI(batch)
    S, T, V = (x.cpu().numpy() for x in eng.engine.one_electron())
    for m, mol in enumerate(batch.mols):
        o, k = batch.bf_off[m], batch.n_bf[m]
        ints = compute_integrals(mol, batch.bases[m], device=0)
        np.testing.assert_allclose(S[o:o + k, o:o + k], np.asarray(ints.S.cpu()), atol=1e-12, rtol=0)
        np.testing.assert_allclose(T[o:o + k, o:o + k], np.asarray(ints.T.cpu()), atol=1e-12, rtol=0)
        np.testing.assert_allclose(V[o:o + k, o:o + k], np.asarray(ints.V.cpu()), atol=1e-11, rtol=0)
    o1 = batch.bf_off[1]
    assert np.all(S[:o1, o1:] == 0.0) and np.all(V[:o1, o1:] == 0.0)
    eng.close()


def test_graph_replay_matches_eager_and_follows_buffer_contents():
    batch = MoleculeBatch(_mols([2, 4, 1]), BASIS)
    eng = BatchedERI(batch)
    rng = np.random.default_rng(9)
    D, J, K = eng.buffers(1)
    D[0].copy_(torch.tensor(_random_block_density(batch, rng), device=DEV))
    gid = eng.capture_jk(D, J, K, "fp64", dens_tau=BATCH_DENS_TAU)
    for trial in range(2):
        D[0].copy_(torch.tensor(_random_block_density(batch, rng), device=DEV))
        J.fill_(float("nan"))
        K.fill_(float("nan"))
        eng.launch(gid)
        J2, K2 = torch.empty_like(J), torch.empty_like(K)
        eng.jk_into(D, J2, K2, "fp64", dens_tau=BATCH_DENS_TAU)
        torch.cuda.synchronize()
        np.testing.assert_allclose(J.cpu().numpy(), J2.cpu().numpy(), atol=1e-11, rtol=0)
        np.testing.assert_allclose(K.cpu().numpy(), K2.cpu().numpy(), atol=1e-11, rtol=0)
    # a new work list (different bra chunking) destroys the graph
    cfg = eng.tuning()
    cfg[:, 1] = 64
    eng.set_tuning(cfg)
    with pytest.raises(ValueError, match="invalidated"):
        eng.launch(gid)
    eng.close()


def test_capture_requires_prebuilt_work_list_and_created_stream():
    batch = MoleculeBatch(_mols([1]), BASIS)
    eng = BatchedERI(batch)
    D, J, K = eng.buffers(1)
    with pytest.raises(ValueError, match="legacy default stream"):
        _abi.call("jqc_graph_begin", eng.engine._ctx, None)
    s = torch.cuda.Stream()
    import ctypes

    sp = ctypes.c_void_p(s.cuda_stream)
    s.wait_stream(torch.cuda.current_stream())
    _abi.call("jqc_graph_begin", eng.engine._ctx, sp)
    with pytest.raises(_abi.JQCError, match="before the capture"):
        eng.jk_into(D, J, K, "fp32", stream=s)  # no FP32 work list yet
    gid = ctypes.c_int(-1)
    rc = eng.engine.lib.jqc_graph_end(eng.engine._ctx, sp, ctypes.byref(gid))
    if rc == 0:
        eng.engine.lib.jqc_graph_destroy(eng.engine._ctx, gid.value)
    torch.cuda.synchronize()
    eng.close()


@pytest.mark.parametrize("threads,persistent,lane_prims", [(64, 1, 64), (256, 0, 1024), (256, 1, 128)])
def test_launch_shapes_give_same_jk(threads, persistent, lane_prims):
    batch = MoleculeBatch(_mols([3, 2]), BASIS)
    eng = BatchedERI(batch)
    rng = np.random.default_rng(4)
    D = torch.tensor(_random_block_density(batch, rng), device=DEV)[None].contiguous()
    J0, K0 = torch.empty_like(D), torch.empty_like(D)
    eng.jk_into(D, J0, K0)
    cfg = eng.tuning()
    assert cfg.shape == (21, 4) and np.all(cfg[:, 0] == 128)
    cfg[:, 0], cfg[:, 1], cfg[:, 2] = threads, lane_prims, persistent
    eng.set_tuning(cfg)
    np.testing.assert_array_equal(eng.tuning(), cfg)
    J, K = torch.empty_like(D), torch.empty_like(D)
    for prec in ("fp64", "mixed"):
        eng.jk_into(D, J, K, prec, mixed_tau=1e-7)
        torch.cuda.synchronize()
        tol = 1e-10 if prec == "fp64" else 1e-6
        np.testing.assert_allclose(J.cpu().numpy(), J0.cpu().numpy(), atol=tol, rtol=0)
        np.testing.assert_allclose(K.cpu().numpy(), K0.cpu().numpy(), atol=tol, rtol=0)
    bad = cfg.copy()
    bad[0, 0] = 96
    with pytest.raises(ValueError, match="threads"):
        eng.set_tuning(bad)
    bad = cfg.copy()
    bad[0, 3] = 1  # (ss|ss) has no column-engine kernel
    with pytest.raises(ValueError, match="engine"):
        eng.set_tuning(bad)
    eng.close()


@pytest.mark.parametrize("engine", [0, 1, 2])
def test_engines_agree_on_high_l_classes(engine):
    """Every engine that can evaluate a class gives the same J/K (FP64 1e-10,
    FP32 split 1e-6)."""
    batch = MoleculeBatch(_mols([3, 2], seed=7), BASIS)
    eng = BatchedERI(batch)
    rng = np.random.default_rng(8)
    D = torch.tensor(_random_block_density(batch, rng), device=DEV)[None].contiguous()
    J0, K0 = torch.empty_like(D), torch.empty_like(D)
    eng.jk_into(D, J0, K0)
    Jm0, Km0 = torch.empty_like(D), torch.empty_like(D)
    eng.jk_into(D, Jm0, Km0, "mixed", mixed_tau=1e-3)
    cfg = eng.tuning()
    from jax_examples_b200.engine import QUARTET_CLASSES

    col = [12, 13, 14, 16, 17, 18, 19, 20]
    for q in range(21):
        L = sum(QUARTET_CLASSES[q])
        ok = {0: L <= 6, 1: q in col, 2: True}[engine]
        if ok:
            cfg[q, 3] = engine
    eng.set_tuning(cfg)
    J, K = torch.empty_like(D), torch.empty_like(D)
    eng.jk_into(D, J, K)
    torch.cuda.synchronize()
    np.testing.assert_allclose(J.cpu().numpy(), J0.cpu().numpy(), atol=1e-10, rtol=0)
    np.testing.assert_allclose(K.cpu().numpy(), K0.cpu().numpy(), atol=1e-10, rtol=0)
    eng.jk_into(D, J, K, "mixed", mixed_tau=1e-3)
    torch.cuda.synchronize()
    np.testing.assert_allclose(J.cpu().numpy(), Jm0.cpu().numpy(), atol=1e-6, rtol=0)
    np.testing.assert_allclose(K.cpu().numpy(), Km0.cpu().numpy(), atol=1e-6, rtol=0)
    eng.close()


def test_autotune_keeps_results_and_uses_cache(tmp_path):
    batch = MoleculeBatch(_mols([4, 2, 1]), BASIS)
    eng = BatchedERI(batch)
    rng = np.random.default_rng(6)
    D = torch.tensor(_random_block_density(batch, rng), device=DEV)[None].contiguous()
    J0, K0 = torch.empty_like(D), torch.empty_like(D)
    eng.jk_into(D, J0, K0)
    cache = str(tmp_path / "tune.txt")
    J, K = torch.empty_like(D), torch.empty_like(D)
    assert eng.autotune(D, J, K, "fp64", dens_tau=0.0, cache_path=cache) is False
    tuned = eng.tuning()
    assert set(np.unique(tuned[:, 0])) <= {64, 128, 256}
    eng.jk_into(D, J, K)
    torch.cuda.synchronize()
    np.testing.assert_allclose(J.cpu().numpy(), J0.cpu().numpy(), atol=1e-10, rtol=0)
    np.testing.assert_allclose(K.cpu().numpy(), K0.cpu().numpy(), atol=1e-10, rtol=0)
    lines = open(cache).read().strip().splitlines()
    assert len(lines) == 1 and len(lines[0].split("\t")[1].split()) == 84
    eng.close()
    eng2 = BatchedERI(batch)
    assert eng2.autotune(D, J, K, "fp64", dens_tau=0.0, cache_path=cache) is True
    np.testing.assert_array_equal(eng2.tuning(), tuned)
    eng2.close()


def test_rhf_batch_energies_and_gradients_match_single_runs():
    mols = _mols([1, 3, 2], seed=11, noise=0.1)
    batch = MoleculeBatch(mols, BASIS)
    cfg = CalcConfig(scf_conv=1e-10, schwarz_tau=1e-12)
    scf = run_rhf_batch(batch, cfg, use_graph=True)
    grads = rhf_gradient_batch(batch, scf)
    assert scf.record["graph"] and scf.record["fock_builds"] >= 2
    for m, mol in enumerate(mols):
        res_b = scf.results[m]
        assert res_b.converged
        ints = compute_integrals(mol, batch.bases[m], device=0, schwarz_tau=1e-12)
        res = run_scf(mol, ints, CalcConfig(scf_conv=1e-10, schwarz_tau=1e-12))
        assert abs(res_b.energy - res.energy) < 1e-8
        g = rhf_gradient(mol, res, batch.bases[m])
        np.testing.assert_allclose(grads[m].cpu().numpy(), g.cpu().numpy(), atol=1e-7, rtol=0)
    scf.engine.close()


def test_bfgs_batch_matches_single_molecule_runs():
    mols = [pb.water_cluster(1, seed=21, noise_angstrom=0.1), pb.water_cluster(2, seed=22, noise_angstrom=0.1)]
    both = optimize_bfgs_batch(mols, BASIS, max_steps=3)
    for m, mol in enumerate(mols):
        alone = optimize_bfgs_batch([mol], BASIS, max_steps=3)[0]
        assert both[m].n_steps == alone.n_steps
        e_b = np.array([e for _, e in both[m].trajectory])
        e_a = np.array([e for _, e in alone.trajectory])
        np.testing.assert_allclose(e_b, e_a, atol=1e-8, rtol=0)
        assert np.all(np.diff(e_b) <= 1e-10)  # Armijo steps never raise the energy


def test_geometry_update_and_molecule_mask_match_fresh_engines():
    """jqc_set_geometry + jqc_molecule_mask in one context give the J/K,
    one-electron integrals and gradient of fresh engines at the new geometry
    (1e-10); masked molecules contribute nothing; the launch tuning
    survives the update."""
    from jax_examples_b200.grad import grad_two_electron

    mols = _mols([2, 1, 3], seed=41, noise=0.05)
    batch = MoleculeBatch(mols, BASIS)
    eng = BatchedERI(batch, schwarz_tau=1e-12)
    tuned = eng.tuning().copy()
    tuned[0, 0] = 64 if tuned[0, 0] != 64 else 256
    eng.set_tuning(tuned)
    rng = np.random.default_rng(42)
    moved = {}
    for m in range(3):  # small displacements, as a BFGS step makes
        xyz = np.asarray(mols[m].coords) + rng.normal(0.0, 0.05, np.asarray(mols[m].coords).shape)
        moved[m] = pb.make_molecule(mols[m].elements, xyz, mols[m].atomic_numbers)
    eng.update_geometry({0: moved[0], 2: moved[2]}, [True, False, True])
    np.testing.assert_array_equal(eng.tuning(), tuned)
    D = torch.tensor(_random_block_density(batch, rng), device=DEV)[None].contiguous()
    J, K = torch.empty_like(D), torch.empty_like(D)
    eng.jk_into(D, J, K)
    S, T, V = eng.engine.one_electron()
    g2 = grad_two_electron(eng.engine, [D[0]], 1.0, 0.5)
    for m in range(3):
        o, k = batch.bf_off[m], batch.n_bf[m]
        blk = (slice(o, o + k), slice(o, o + k))
        if m == 1:  # left out: no quartets, no forces
            assert float(J[0][blk].abs().max()) == 0.0 and float(K[0][blk].abs().max()) == 0.0
            assert float(batch.atoms(g2, m).abs().max()) == 0.0
            continue
        mol = moved[m]
        np.testing.assert_allclose(np.asarray(batch.mols[m].coords), np.asarray(mol.coords), atol=0)
        single = DirectERI(pb.build_basis_set(mol, BASIS), mol, device=0, schwarz_tau=1e-12)
        Js, Ks = single.jk(D[0][blk].contiguous())
        np.testing.assert_allclose(J[0][blk].cpu().numpy(), Js.cpu().numpy(), atol=1e-10, rtol=0)
        np.testing.assert_allclose(K[0][blk].cpu().numpy(), Ks.cpu().numpy(), atol=1e-10, rtol=0)
        Ss, Ts, Vs = single.one_electron()
        np.testing.assert_allclose(S[blk].cpu().numpy(), Ss.cpu().numpy(), atol=1e-12, rtol=0)
        np.testing.assert_allclose(V[blk].cpu().numpy(), Vs.cpu().numpy(), atol=1e-11, rtol=0)
        gs = grad_two_electron(single, [D[0][blk].contiguous()], 1.0, 0.5)
        np.testing.assert_allclose(batch.atoms(g2, m).cpu().numpy(), gs.cpu().numpy(), atol=1e-10, rtol=0)
        single.close()
    eng.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_molecule_activity_compacts_builds(prec):
    """jqc_set_molecule_activity: with molecule 1 of three flagged inactive
    the build equals the full build on the active molecules' blocks (1e-12)
    and leaves molecule 1's blocks zero; flags rewritten in place between two
    replays of one captured graph select other molecules."""
    mols = _mols([2, 1, 3], seed=51, noise=0.05)
    batch = MoleculeBatch(mols, BASIS)
    eng = BatchedERI(batch, schwarz_tau=1e-12)
    rng = np.random.default_rng(52)
    D = torch.tensor(_random_block_density(batch, rng), device=DEV)[None].contiguous()
    J0, K0 = torch.empty_like(D), torch.empty_like(D)
    eng.jk_into(D, J0, K0, prec, 1e-4)
    flags = torch.tensor([1, 0, 1], dtype=torch.int32, device=DEV)
    eng.engine.set_molecule_activity(flags)

    def check(J, K, active):
        for m in range(3):
            o, k = batch.bf_off[m], batch.n_bf[m]
            blk = (slice(o, o + k), slice(o, o + k))
            if active[m]:
                np.testing.assert_allclose(J[0][blk].cpu().numpy(), J0[0][blk].cpu().numpy(), atol=1e-12, rtol=0)
                np.testing.assert_allclose(K[0][blk].cpu().numpy(), K0[0][blk].cpu().numpy(), atol=1e-12, rtol=0)
            else:
                assert float(J[0][blk].abs().max()) == 0.0 and float(K[0][blk].abs().max()) == 0.0

    J, K = torch.empty_like(D), torch.empty_like(D)
    eng.jk_into(D, J, K, prec, 1e-4)
    check(J, K, [1, 0, 1])
    gid = eng.capture_jk(D, J, K, prec, 1e-4, 0.0)
    flags.copy_(torch.tensor([0, 1, 1], dtype=torch.int32))
    J.fill_(float("nan"))
    eng.launch(gid)
    torch.cuda.synchronize()
    check(J, K, [0, 1, 1])
    eng.engine.set_molecule_activity(None)
    eng.jk_into(D, J, K, prec, 1e-4)
    check(J, K, [1, 1, 1])
    eng.close()


def _set_grad_engines(eng, engine, classes):
    for q in classes:
        _abi.call("jqc_set_grad_engine", eng._ctx, q, engine)


def test_gradient_engines_agree():
    """The register (one or two sides), row and warp engines of the
    ERI-derivative adjoint give the same two-electron gradient (1e-10
    Eh/bohr) wherever they overlap."""
    from jax_examples_b200.grad import grad_two_electron

    mol = pb.water_cluster(3, seed=12, noise_angstrom=0.1)
    bs = pb.build_basis_set(mol, BASIS)
    eng = DirectERI(bs, mol, device=0, schwarz_tau=1e-12)
    rng = np.random.default_rng(13)
    n = bs.n_basis
    a = rng.standard_normal((n, n)) * 0.05
    D = torch.tensor(a + a.T, device=DEV)
    engines = np.zeros(21, dtype=np.int32)
    _abi.call("jqc_get_grad_engine", eng._ctx, engines.ctypes.data_as(_abi._ip))
    g0 = grad_two_electron(eng, [D], 1.0, 0.5)
    row = [11, 12, 13, 14, 15, 16, 17, 18, 19, 20]
    _set_grad_engines(eng, 2, range(21))  # warp engine everywhere
    g_warp = grad_two_electron(eng, [D], 1.0, 0.5)
    np.testing.assert_allclose(g_warp.cpu().numpy(), g0.cpu().numpy(), atol=1e-10, rtol=0)
    _set_grad_engines(eng, 1, row)  # row engine where it exists
    g_row = grad_two_electron(eng, [D], 1.0, 0.5)
    np.testing.assert_allclose(g_row.cpu().numpy(), g0.cpu().numpy(), atol=1e-10, rtol=0)
    _set_grad_engines(eng, 0, [11, 15])  # register kernels for the L <= 4 row classes
    g_reg = grad_two_electron(eng, [D], 1.0, 0.5)
    np.testing.assert_allclose(g_reg.cpu().numpy(), g0.cpu().numpy(), atol=1e-10, rtol=0)
    reg = [q for q in range(21) if q not in (12, 13, 14, 16, 17, 18, 19, 20)]
    _set_grad_engines(eng, 3, reg)  # register kernels, bra and ket forces in separate parts
    g_split = grad_two_electron(eng, [D], 1.0, 0.5)
    np.testing.assert_allclose(g_split.cpu().numpy(), g0.cpu().numpy(), atol=1e-10, rtol=0)
    with pytest.raises(ValueError, match="engine"):
        _abi.call("jqc_set_grad_engine", eng._ctx, 0, 1)  # (ss|ss) has no row kernel
    with pytest.raises(ValueError, match="engine"):
        _abi.call("jqc_set_grad_engine", eng._ctx, 13, 3)  # (dp|ds): L = 5, no register kernel
    eng.close()


def test_rhf_batch_mixed_policy_matches_fp64():
    """The batched mixed path (incremental screened builds, FP64 tail, graphs)
    converges every molecule to the FP64 energy within 1e-6 Eh and its
    screened gradient to the FP64 gradient within 1e-5 Eh/bohr."""
    from jax_examples_b200.batch import MIXED_GRAD_TAU

    mols = _mols([2, 4, 1], seed=31, noise=0.1)
    batch = MoleculeBatch(mols, BASIS)
    plain = run_rhf_batch(batch, CalcConfig(scf_conv=1e-9, schwarz_tau=1e-12, incremental=False))
    g_plain = rhf_gradient_batch(batch, plain)
    mixed = run_rhf_batch(batch, CalcConfig(scf_conv=1e-9, schwarz_tau=1e-12, precision="mixed", incremental=True))
    g_mixed = rhf_gradient_batch(batch, mixed, dens_tau=MIXED_GRAD_TAU)
    rec = mixed.record
    assert rec["builds_mixed"] > 0 and rec["builds_fp64"] >= 2 and rec["incremental_builds"] > 0
    for m in range(len(mols)):
        assert mixed.results[m].converged
        assert abs(mixed.results[m].energy - plain.results[m].energy) < 1e-6
        np.testing.assert_allclose(g_mixed[m].cpu().numpy(), g_plain[m].cpu().numpy(), atol=1e-5, rtol=0)
    plain.engine.close()
    mixed.engine.close()
