"""drop_in.install() against the reference's own SCF drivers (CPU).

Runs only where the reference checkout can be imported (through the test
shim); the GPU box does not have it.  The direct engine is replaced by a
fake backed by the CPU oracle, so this checks the plumbing: the reference's
run_rhf/run_uhf (with DIIS and the UHF alpha-repulsion guess) call the
patched Fock builders and reach the reference's own energies."""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest
import torch

import oracle
from conftest import GOLDEN, ROOT

def _reference_root() -> str:
    """The reference checkout: ``JQC_REFERENCE_ROOT``, else the parent of an
    importable ``jax_qc`` package; empty when neither exists."""
    root = os.environ.get("JQC_REFERENCE_ROOT", "")
    if root:
        return root
    import importlib.util

    spec = importlib.util.find_spec("jax_qc") if "jax_qc" not in sys.modules else None
    if spec is not None and spec.origin:
        return os.path.dirname(os.path.dirname(spec.origin))
    return ""


REF = _reference_root()
pytestmark = pytest.mark.skipif(not REF or not os.path.isdir(os.path.join(REF, "jax_qc")),
                                reason="reference checkout not available (set JQC_REFERENCE_ROOT)")


class FakeDirect:
    """Stands in for DirectERI on CPU: J/K from the oracle's dense tensor."""

    def __init__(self, eri):
        self.eri = eri
        self.device = torch.device("cpu")
        self.n_basis = eri.shape[0]
        self.calls = 0

    def jk(self, D, precision="fp64", mixed_tau=1e-7, dens_tau=0.0):
        self.calls += 1
        D = D.cpu().numpy()
        if D.ndim == 2:
            J, K = oracle.jk_from_tensor(D, self.eri)
            return torch.tensor(J), torch.tensor(K)
        out = [oracle.jk_from_tensor(d, self.eri) for d in D]
        return torch.tensor(np.array([o[0] for o in out])), torch.tensor(np.array([o[1] for o in out]))


@pytest.fixture(scope="module")
def ref():
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden", "shim"))
    sys.path.insert(0, REF)
    import jax_qc
    from jax_qc.scf import diis as rdiis

    def _push(history, F, e):
        if history.size < history.max_size:
            fl = np.array(history.fock_list)
            el = np.array(history.error_list)
            fl[history.size] = F
            el[history.size] = e
            return history.replace(fock_list=fl, error_list=el, size=history.size + 1)
        fl = np.concatenate([history.fock_list[1:], F[None]], axis=0)
        el = np.concatenate([history.error_list[1:], e[None]], axis=0)
        return history.replace(fock_list=fl, error_list=el)

    rdiis._push = _push
    from jax_examples_b200 import drop_in

    names = drop_in.install(jax_qc)
    yield jax_qc, names
    drop_in.uninstall()


@pytest.mark.parametrize("tag", ["water_synsto3g", "water_cation_synsto3g_uhf", "water_sto3g",
                                 "water_cation_sto3g_uhf"])
def test_reference_scf_through_drop_in(ref, golden, tag):
    jax_qc, names = ref
    assert "jax_qc.scf.rhf.build_fock_rhf" in names and "jax_qc.scf.uhf.build_fock_uhf" in names
    from jax_qc.core.types import CalcConfig, IntegralSet

    g = golden(tag)
    mol = g.molecule()
    from jax_qc.core.types import make_molecule

    rmol = make_molecule(elements=mol.elements, coords=np.asarray(mol.coords), atomic_numbers=np.asarray(mol.atomic_numbers),
                         charge=mol.charge, spin=mol.spin)
    fake = FakeDirect(oracle.eri_tensor(g.basis(), mode=0))
    a = g.arr
    ints = IntegralSet(S=a["S"], T=a["T"], V=a["V"], H_core=a["T"] + a["V"], ERI=fake, E_nuc=g.rec["E_nuc"])
    res = jax_qc.run_scf(rmol, ints, CalcConfig(method="uhf" if mol.spin else "rhf", scf_conv=1e-10))
    assert fake.calls > 3
    assert abs(float(res.energy) - g.rec["energy"]) < 1e-9


def test_gradient_and_bfgs_callers_are_rebound(ref):
    """rhf_gradient is rebound where the reference imported it by name
    (grad/interface.py:17, geomopt/optimizer.py:30, geomopt/hessian.py:21),
    so the reference's BFGS and FD Hessian call the analytic gradient."""
    jax_qc, names = ref
    import importlib

    from jax_examples_b200 import drop_in

    for mod in ("jax_qc.grad.rhf_grad", "jax_qc.grad.interface", "jax_qc.geomopt.optimizer",
                "jax_qc.geomopt.hessian"):
        assert f"{mod}.rhf_gradient" in names
        assert importlib.import_module(mod).rhf_gradient is drop_in.rhf_gradient
