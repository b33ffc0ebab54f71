"""Install the B200 engine behind an imported ``jax_qc`` package.

``install(jax_qc)`` rebinds, in every module that imported them by name, the
reference's two-electron entry points to this package's device path:

* ``jax_qc.integrals.interface.compute_integrals`` (``interface.py:26-67``):
  S/T/V on the device, ``ERI`` = a :class:`DirectERI` handle (the dense
  tensor of ``eri.py:69-105`` is never formed);
* ``jax_qc.integrals.eri.compute_eri_tensor`` (``eri.py:69``): the dense
  tensor from the device kernels, as a host array;
* ``jax_qc.scf.fock.build_fock_rhf`` / ``build_fock_uhf`` (``fock.py:41-79``)
  and their by-name imports in ``scf/rhf.py:37`` and ``scf/uhf.py:51``;
* ``jax_qc.scf.guess.core_guess_uhf`` (its inlined J/K, ``guess.py:87-88``);
* ``jax_qc.grad.rhf_grad.rhf_gradient`` (``rhf_grad.py:106-211``) and its
  by-name imports in ``grad/interface.py:17``, ``geomopt/optimizer.py:30``
  and ``geomopt/hessian.py:21``: the analytic gradient (ERI-derivative
  adjoint kernel, one-electron derivative kernels) in place of the finite
  differences of whole integral sets, so the reference's BFGS
  (``optimizer.py:79-209``) and FD Hessian run on it unchanged.

Matrices are handed back in the caller's array type (NumPy, or JAX arrays
when ``jax`` is importable: a DLPack hand-off of the device tensor), so the
reference's DIIS, diagonalization and energy code runs unchanged.
``uninstall()`` restores the originals.
"""

from __future__ import annotations

import sys
from typing import Dict, Optional, Tuple

import numpy as np
import torch

from .engine import DirectERI
from .fock import _is_direct

_SAVED: Dict[Tuple[str, str], object] = {}
_STATE = {"device": None, "precision": "fp64", "schwarz_tau": 1e-13}


def _to_host(x):
    """Device tensor -> the reference's array type (jax.numpy if real JAX is
    present, else NumPy)."""
    if not torch.is_tensor(x):
        return x
    jnp = sys.modules.get("jax.numpy")
    if jnp is not None and hasattr(jnp, "from_dlpack"):
        try:
            return jnp.from_dlpack(x.contiguous())
        except Exception:
            pass
    return x.detach().cpu().numpy()


def _dev(x, eng):
    return torch.as_tensor(np.asarray(x), dtype=torch.float64, device=eng.device)


def compute_integrals(mol, basis, timer=None):
    """Drop-in for ``jax_qc.integrals.interface.compute_integrals``."""
    from .integrals import compute_integrals as ours

    ref_types = sys.modules.get("jax_qc.core.types")
    ints = ours(mol, basis, timer=timer, device=_STATE["device"], schwarz_tau=_STATE["schwarz_tau"])
    fields = dict(S=_to_host(ints.S), T=_to_host(ints.T), V=_to_host(ints.V), H_core=_to_host(ints.H_core),
                  ERI=ints.ERI, E_nuc=ints.E_nuc)
    if ref_types is not None and hasattr(ref_types, "IntegralSet"):
        return ref_types.IntegralSet(**fields)
    return ints.replace(**fields)


def compute_eri_tensor(basis):
    """Drop-in for ``jax_qc.integrals.eri.compute_eri_tensor``."""
    from .integrals import compute_eri_tensor as ours

    return _to_host(ours(basis, device=_STATE["device"]))


def build_fock_rhf(H_core, D, ERI):
    """Drop-in for ``jax_qc.scf.fock.build_fock_rhf``."""
    if not _is_direct(ERI):
        return _SAVED[("jax_qc.scf.fock", "build_fock_rhf")](H_core, D, ERI)
    J, K = ERI.jk(_dev(D, ERI), precision=_STATE["precision"])
    return _to_host(_dev(H_core, ERI) + J - 0.5 * K)


def build_fock_uhf(H_core, D_alpha, D_beta, ERI):
    """Drop-in for ``jax_qc.scf.fock.build_fock_uhf``."""
    if not _is_direct(ERI):
        return _SAVED[("jax_qc.scf.fock", "build_fock_uhf")](H_core, D_alpha, D_beta, ERI)
    J, K = ERI.jk(torch.stack([_dev(D_alpha, ERI), _dev(D_beta, ERI)]), precision=_STATE["precision"])
    H = _dev(H_core, ERI)
    Jt = J[0] + J[1]
    return _to_host(H + Jt - K[0]), _to_host(H + Jt - K[1])


def core_guess_uhf(H_core, X, n_alpha, n_beta, ERI):
    """Drop-in for ``jax_qc.scf.guess.core_guess_uhf`` (guess.py:42-115): the
    same guess with its J/K from the direct engine."""
    orig = _SAVED[("jax_qc.scf.guess", "core_guess_uhf")]
    if not _is_direct(ERI):
        return orig(H_core, X, n_alpha, n_beta, ERI)
    return orig(H_core, X, n_alpha, n_beta, _JKProxy(ERI))


class _JKProxy:
    """Lets the reference's inlined ``einsum('ls,mnls->mn', D, ERI)`` /
    ``einsum('ls,msln->mn', D, ERI)`` in core_guess_uhf run on the engine."""

    def __init__(self, eng: DirectERI):
        self.eng = eng


def _patched_einsum(orig):
    def einsum(spec, *ops, **kw):
        if len(ops) == 2 and isinstance(ops[1], _JKProxy) and spec in ("ls,mnls->mn", "ls,msln->mn"):
            J, K = ops[1].eng.jk(_dev(ops[0], ops[1].eng), precision=_STATE["precision"])
            return _to_host(J if spec == "ls,mnls->mn" else K)
        return orig(spec, *ops, **kw)

    return einsum


def rhf_gradient(mol, result, basis_name: str = "sto-3g", step_size: float = 1e-4):
    """Drop-in for ``jax_qc.grad.rhf_grad.rhf_gradient`` (same signature;
    ``step_size`` is unused: the gradient is analytic)."""
    from .grad import rhf_gradient as ours

    eng = getattr(result, "ERI", None)
    if not isinstance(eng, DirectERI):
        build = sys.modules.get("jax_qc.basis.build")
        if build is None:
            import importlib

            build = importlib.import_module("jax_qc.basis.build")
        eng = DirectERI(build.build_basis_set(mol, basis_name), mol, device=_STATE["device"],
                        schwarz_tau=_STATE["schwarz_tau"])
    return _to_host(ours(mol, result, engine=eng))


_TARGETS = [
    ("jax_qc.integrals.interface", "compute_integrals", compute_integrals),
    ("jax_qc", "compute_integrals", compute_integrals),
    ("jax_qc.io.input_parser", "compute_integrals", compute_integrals),
    ("jax_qc.grad.rhf_grad", "compute_integrals", compute_integrals),
    ("jax_qc.grad.numerical_grad", "compute_integrals", compute_integrals),
    ("jax_qc.integrals.eri", "compute_eri_tensor", compute_eri_tensor),
    ("jax_qc.scf.fock", "build_fock_rhf", build_fock_rhf),
    ("jax_qc.scf.fock", "build_fock_uhf", build_fock_uhf),
    ("jax_qc.scf.rhf", "build_fock_rhf", build_fock_rhf),
    ("jax_qc.scf.uhf", "build_fock_uhf", build_fock_uhf),
    ("jax_qc.scf.guess", "core_guess_uhf", core_guess_uhf),
    ("jax_qc.scf.uhf", "core_guess_uhf", core_guess_uhf),
    ("jax_qc.grad.rhf_grad", "rhf_gradient", rhf_gradient),
    ("jax_qc.grad.interface", "rhf_gradient", rhf_gradient),
    ("jax_qc.geomopt.optimizer", "rhf_gradient", rhf_gradient),
    ("jax_qc.geomopt.hessian", "rhf_gradient", rhf_gradient),
]


def install(jax_qc=None, device: Optional[int] = None, precision: str = "fp64", schwarz_tau: float = 1e-13):
    """Rebind the reference's two-electron entry points (see module doc).

    ``jax_qc`` is the imported reference package (imported here if None)."""
    if jax_qc is None:
        import jax_qc  # noqa: F401
    import importlib

    _STATE.update(device=device, precision=precision, schwarz_tau=schwarz_tau)
    for modname, attr, fn in _TARGETS:
        try:
            mod = importlib.import_module(modname)
        except ImportError:
            continue
        if not hasattr(mod, attr):
            continue
        key = (modname, attr)
        if key not in _SAVED:
            _SAVED[key] = getattr(mod, attr)
        setattr(mod, attr, fn)
    guess = sys.modules.get("jax_qc.scf.guess")
    if guess is not None and ("guess.jnp", "einsum") not in _SAVED:
        jnp_mod = guess.jnp
        _SAVED[("guess.jnp", "einsum")] = (jnp_mod, jnp_mod.einsum)
        guess.jnp = _JnpShim(jnp_mod)
    return sorted(f"{m}.{a}" for m, a in _SAVED if not m.startswith("guess."))


class _JnpShim:
    """jax.numpy seen by scf/guess.py with einsum routed to the engine."""

    def __init__(self, mod):
        self._mod = mod
        self.einsum = _patched_einsum(mod.einsum)

    def __getattr__(self, name):
        return getattr(self._mod, name)


def uninstall():
    import importlib

    for (modname, attr), orig in list(_SAVED.items()):
        if modname == "guess.jnp":
            guess = sys.modules.get("jax_qc.scf.guess")
            if guess is not None:
                guess.jnp = orig[0]
            continue
        try:
            setattr(importlib.import_module(modname), attr, orig)
        except ImportError:
            pass
    _SAVED.clear()
