"""The allocation-free J/K entry point (jqc_jk_noalloc) against jqc_jk.

Callers such as a Fock builder running inside a JAX/XLA program cannot
allocate device memory at build time (XLA owns and pre-reserves the GPU's
memory), so they build the work list once at set-up with jqc_jk and then use
jqc_jk_noalloc, whose only scratch is a static device array.  This file is
named so pytest collects it last; it builds its own engine and passes both
alone and after the other tests.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from jax_examples_b200 import DirectERI, _abi
from jax_examples_b200 import basis as pb

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _call(name, eng, D, J, K, prec, mixed_tau, dens_tau):
    stream = ctypes.c_void_p(torch.cuda.current_stream(eng.device).cuda_stream)
    _abi.call(name, eng._ctx, D.shape[0], _ptr(D), _ptr(J), _ptr(K), _abi.PREC[prec], mixed_tau, dens_tau, stream)


@pytest.mark.parametrize("prec,dens_tau", [("fp64", 1e-11), ("mixed", 0.0)])
def test_noalloc_matches_jk_twice(prec, dens_tau):
    mol = pb.water_cluster(3, seed=5)
    bs = pb.build_basis_set(mol, "6-31g*")
    eng = DirectERI(bs, mol, device=0, schwarz_tau=1e-12)
    n = bs.n_basis
    rng = np.random.default_rng(11)
    Dn = rng.standard_normal((2, n, n)) * 0.05
    D = torch.tensor(Dn + Dn.transpose(0, 2, 1), device="cuda:0").contiguous()
    J0 = torch.empty_like(D)
    K0 = torch.empty_like(D)
    # set-up call of the allocating entry point: builds the work list
    _call("jqc_jk", eng, D, J0, K0, prec, 1e-7, dens_tau)
    for _ in range(2):  # two calls in a row share (and fully rewrite) the scratch
        J = torch.full_like(D, float("nan"))
        K = torch.full_like(D, float("nan"))
        _call("jqc_jk_noalloc", eng, D, J, K, prec, 1e-7, dens_tau)
        torch.cuda.synchronize()
        np.testing.assert_allclose(J.cpu().numpy(), J0.cpu().numpy(), atol=1e-10, rtol=0)
        np.testing.assert_allclose(K.cpu().numpy(), K0.cpu().numpy(), atol=1e-10, rtol=0)
    eng.close()


def test_noalloc_requires_prebuilt_work_list():
    mol = pb.water_cluster(1, seed=0)
    bs = pb.build_basis_set(mol, "6-31g*")
    eng = DirectERI(bs, mol, device=0, schwarz_tau=1e-12)
    n = bs.n_basis
    D = torch.eye(n, dtype=torch.float64, device="cuda:0")[None].contiguous()
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    with pytest.raises(_abi.JQCError, match="work list"):
        _call("jqc_jk_noalloc", eng, D, J, K, "fp32", 1e-7, 0.0)
    eng.close()


def test_noalloc_leaves_device_memory_untouched():
    """After the set-up call, repeated jqc_jk_noalloc calls change the
    device's free memory by nothing (cudaMemGetInfo before and after)."""
    mol = pb.water_cluster(2, seed=9)
    bs = pb.build_basis_set(mol, "6-31g*")
    eng = DirectERI(bs, mol, device=0, schwarz_tau=1e-12)
    n = bs.n_basis
    D = torch.eye(n, dtype=torch.float64, device="cuda:0")[None].contiguous() * 0.1
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    _call("jqc_jk", eng, D, J, K, "fp64", 1e-7, 1e-11)
    _call("jqc_jk_noalloc", eng, D, J, K, "fp64", 1e-7, 1e-11)  # first call on the device: address look-up
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):
        _call("jqc_jk_noalloc", eng, D, J, K, "fp64", 1e-7, 1e-11)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
    eng.close()


def test_noalloc_rejects_more_shells_than_the_static_scratch():
    """52 waters in 6-31G* have 520 shells, more than the 512 the static
    scratch holds: the call fails with JQC_ERR_TOO_LARGE before it looks
    for a work list or launches anything."""
    mol = pb.water_cluster(52, seed=0)
    bs = pb.build_basis_set(mol, "6-31g*")
    assert len(bs.shells) == 520
    eng = DirectERI(bs, mol, device=0, schwarz_tau=1e-10)
    n = bs.n_basis
    D = torch.zeros((1, n, n), dtype=torch.float64, device="cuda:0")
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    with pytest.raises(_abi.JQCTooLarge, match="static scratch"):
        _call("jqc_jk_noalloc", eng, D, J, K, "fp64", 1e-7, 0.0)
    eng.close()
