"""Host logic of the batched path (CPU only): the batch layout, and the BFGS
walker pinned to the reference optimizer's own trajectories
(tests/golden/bfgs_model.json, made by gen_bfgs_golden.py from
jax_qc/geomopt/optimizer.py with its energy/gradient replaced by an analytic
pair potential)."""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

from jax_examples_b200 import basis as pb
from jax_examples_b200 import batch as jb
from jax_examples_b200.core import make_molecule

from conftest import GOLDEN

import importlib.util

_spec = importlib.util.spec_from_file_location("gen_bfgs_golden", os.path.join(GOLDEN, "gen_bfgs_golden.py"))
_gen = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_gen)
model_energy_gradient = _gen.model_energy_gradient


def _cases():
    return json.load(open(os.path.join(GOLDEN, "bfgs_model.json")))["cases"]


def _mol(rec):
    return make_molecule(tuple(rec["elements"]), np.array(rec["coords"]), np.array(rec["Z"]))


def _drive(walker, r0):
    """Run one walker to completion against the model potential."""
    x = walker.send(None)
    while True:
        e, g = model_energy_gradient(x, r0)
        try:
            x = walker.send((e, g))
        except StopIteration as stop:
            return stop.value


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_bfgs_walker_matches_reference_trajectory(idx):
    rec = _cases()[idx]
    r0 = np.array(rec["r0"])
    res = _drive(jb._bfgs_walker(_mol(rec), rec["max_steps"], rec["grad_tol"], 1e-6, 0.3), r0)
    assert res.converged == rec["converged"]
    assert res.n_steps == rec["n_steps"]
    np.testing.assert_allclose([e for _, e in res.trajectory], rec["trajectory_energies"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(np.asarray(res.molecule.coords), np.array(rec["final_coords"]), rtol=0, atol=1e-10)
    np.testing.assert_allclose(res.gradient, np.array(rec["final_gradient"]), rtol=0, atol=1e-10)


def test_batched_bfgs_rounds_equal_independent_runs(monkeypatch):
    """Batching the evaluations of several walkers changes none of them."""
    recs = _cases()
    mols = [_mol(r) for r in recs]
    by_natoms = {len(m.atomic_numbers): np.array(r["r0"]) for m, r in zip(mols, recs)}
    calls = []

    class FakeEvaluator:
        """Stands in for the device evaluator: the model potential per molecule."""

        def __init__(self, mols_, basis, config, *a):
            self.mols = mols_
            self.rounds = 0

        def __call__(self, coords):
            calls.append(len(coords))
            self.rounds += 1
            return {i: model_energy_gradient(np.asarray(c), by_natoms[len(self.mols[i].atomic_numbers)])
                    for i, c in coords.items()}

        def close(self):
            pass

    monkeypatch.setattr(jb, "_BatchEvaluator", FakeEvaluator)
    res = jb.optimize_bfgs_batch(mols, "model", max_steps=25, grad_tol=1e-5)
    for m, rec in zip(res, recs):
        assert m.n_steps == rec["n_steps"] and m.converged == rec["converged"]
        np.testing.assert_allclose([e for _, e in m.trajectory], rec["trajectory_energies"], rtol=0, atol=1e-12)
    # one batch per round: the first round holds all three molecules, later
    # rounds only the unfinished ones
    assert calls[0] == 3 and max(calls) == 3 and calls[-1] == 1


def test_molecule_batch_layout():
    mols = [pb.water_cluster(n, seed=n) for n in (2, 1, 3)]
    b = jb.MoleculeBatch(mols, "6-31g*")
    assert b.n_bf == [38, 19, 57] and b.bf_off == [0, 38, 57] and b.n_basis == 114
    assert b.atom_off == [0, 6, 9] and b.n_atoms == [6, 3, 9]
    np.testing.assert_array_equal(b.mol_of_atom, [0] * 6 + [1] * 3 + [2] * 9)
    assert len(b.basis.shells) == sum(len(x.shells) for x in b.bases)
    # shells keep their centres and point at their molecule's atoms
    for m, bs in enumerate(b.bases):
        for sh in bs.shells:
            assert 0 <= int(sh.atom_index) < b.n_atoms[m]
    atoms = np.array([int(sh.atom_index) for sh in b.basis.shells])
    assert np.all(np.diff(b.mol_of_atom[atoms]) >= 0)
    np.testing.assert_allclose(b.coords[b.atom_off[2]:], np.asarray(mols[2].coords))
    M = np.arange(b.n_basis ** 2, dtype=float).reshape(b.n_basis, b.n_basis)
    import torch

    blk = b.block(torch.tensor(M), 1)
    np.testing.assert_array_equal(blk.numpy(), M[38:57, 38:57])
    with pytest.raises(ValueError):
        jb.MoleculeBatch([], "6-31g*")


def test_pooled_eigensolver_matches_per_matrix_eigh():
    """The host eigensolver of the batched SCF: per member X^T F X solved on
    the worker pool equals a plain eigh, for all members and for a subset
    (the others come back as eps = 0, C = X)."""
    import torch

    rng = np.random.default_rng(7)
    n_threads = torch.get_num_threads()

    class G:
        pass

    groups, Fs = [], []
    for n, m in [(19, 3), (38, 1), (57, 4)]:
        S = rng.standard_normal((m, n, n))
        S = S @ S.transpose(0, 2, 1) / n + np.eye(n)
        w, U = np.linalg.eigh(S)
        g = G()
        g.X = torch.tensor(U * (1.0 / np.sqrt(w))[:, None, :] @ U.transpose(0, 2, 1))
        F = rng.standard_normal((m, n, n))
        groups.append(g)
        Fs.append(torch.tensor(F + F.transpose(0, 2, 1)))
    for active in (None, [np.array([True, False, True]), np.array([False]), np.array([False, True, True, False])]):
        out = jb._diag_all(groups, Fs, active)
        for k, (g, F) in enumerate(zip(groups, Fs)):
            eps, C = out[k]
            for i in range(F.shape[0]):
                if active is not None and not active[k][i]:
                    assert torch.all(eps[i] == 0) and torch.equal(C[i], g.X[i])
                    continue
                A = g.X[i].T @ F[i] @ g.X[i]
                e_ref, _ = torch.linalg.eigh(A)
                torch.testing.assert_close(eps[i], e_ref, rtol=0, atol=1e-12)
                # C^T F C = diag(eps) and C^T S C = 1 with S = X^-2
                torch.testing.assert_close(C[i].T @ F[i] @ C[i], torch.diag(eps[i]), rtol=0, atol=1e-10)
                Xi = torch.linalg.inv(g.X[i])
                torch.testing.assert_close(C[i].T @ (Xi @ Xi) @ C[i], torch.eye(F.shape[-1], dtype=F.dtype),
                                           rtol=0, atol=1e-10)
    assert torch.get_num_threads() == n_threads  # the caller's solver threads are left as they were


def test_batch_density_scatter_matches_block_copies():
    """_BatchFock writes the active molecules' densities (or density changes)
    into the batch buffer with one indexed copy: the same matrix as one
    block copy per molecule, zero outside the active blocks."""
    import torch

    mols = [pb.water_cluster(n, seed=5 + n) for n in (1, 2, 1)]
    batch = jb.MoleculeBatch(mols, "sto-3g")
    N = batch.n_basis
    fb = jb._BatchFock.__new__(jb._BatchFock)
    fb.batch = batch
    fb.D = torch.full((1, N, N), 7.0, dtype=torch.float64)
    fb._flat_idx = {}
    g = torch.Generator().manual_seed(3)
    dens = {m: torch.rand((batch.n_bf[m],) * 2, generator=g, dtype=torch.float64) for m in (2, 0)}
    prev = {m: torch.rand((batch.n_bf[m],) * 2, generator=g, dtype=torch.float64) for m in (2, 0)}
    for p in (None, prev):
        fb._scatter(dens, p)
        ref = torch.zeros((N, N), dtype=torch.float64)
        for m, d in dens.items():
            batch.block(ref, m).copy_(d if p is None else d - p[m])
        assert torch.equal(fb.D[0], ref)
    fb._scatter({})
    assert float(fb.D.abs().max()) == 0.0
