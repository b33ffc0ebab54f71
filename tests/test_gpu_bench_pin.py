"""The benchmarked Fock build pinned at its own configuration.

bench.py times the direct FP64 J/K build of (H2O)16 in 6-31G* (304
Cartesian functions) with Schwarz screening at 1e-12 and primitive-pair
dropping at 1e-20.  Here that exact build, from the core-guess density, is
compared with the oracle's *unscreened* direct digestion of every canonical
shell quartet (``scf/fock.py:31-38`` over ``eri.py:89-104``'s quartet
loop): J and K within 1e-10.  The same for (H2O)8 in 6-31G** (200
functions).  The oracle runs on all host cores (OpenMP), in chunks of bra
shell pairs whose J/K add up.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from jax_examples_b200 import DirectERI
from jax_examples_b200 import basis as pb

pytestmark = pytest.mark.gpu


def _core_guess(eng, n_occ):
    S, T, V = eng.one_electron()
    w, U = torch.linalg.eigh(S)
    X = (U * (1.0 / torch.sqrt(w))[None, :]) @ U.T
    _, Cp = torch.linalg.eigh(X.T @ (T + V) @ X)
    C = X @ Cp
    return (2.0 * C[:, :n_occ] @ C[:, :n_occ].T).contiguous()


def _oracle_jk_all_quartets(bs, D, chunk_pairs=256):
    """Unscreened J/K over all canonical quartets (ij|kl), ij >= kl."""
    pk = oracle.Packed(bs)
    ns = pk.n_shell
    ii, jj = np.tril_indices(ns)  # pair p = (ii[p], jj[p]) with i >= j, in row order
    n_pairs = len(ii)
    J = np.zeros((pk.n, pk.n))
    K = np.zeros((pk.n, pk.n))
    for p0 in range(0, n_pairs, chunk_pairs):
        p1 = min(n_pairs, p0 + chunk_pairs)
        bra = np.repeat(np.arange(p0, p1), np.arange(p0, p1) + 1)
        ket = np.concatenate([np.arange(p + 1) for p in range(p0, p1)])
        q = np.stack([ii[bra], jj[bra], ii[ket], jj[ket]], axis=1).astype(np.int32)
        Jc, Kc = oracle.jk_quartets(pk, D, q, mode=1)
        J += Jc
        K += Kc
    return J, K


@pytest.mark.parametrize("n_waters,basis", [(16, "6-31g*"), (8, "6-31g**")])
def test_benchmarked_build_vs_unscreened_oracle(n_waters, basis):
    mol = pb.water_cluster(n_waters, seed=0)
    bs = pb.build_basis_set(mol, basis)
    eng = DirectERI(bs, mol, device=0, schwarz_tau=1e-12, prim_tau=1e-20)  # bench.py's settings
    D = _core_guess(eng, mol.n_electrons // 2)
    J, K = eng.jk(D)
    Jr, Kr = _oracle_jk_all_quartets(bs, D.cpu().numpy())
    np.testing.assert_allclose(J.cpu().numpy(), Jr, atol=1e-10, rtol=0)
    np.testing.assert_allclose(K.cpu().numpy(), Kr, atol=1e-10, rtol=0)
    eng.close()
