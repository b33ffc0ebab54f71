"""Device-resident two-electron engine: the handle the drop-in passes around.

``DirectERI`` owns one libjqc context: the basis and nuclei uploaded once,
shell-pair data and Schwarz bounds built on the device, and the class-sorted
work lists.  It is what ``compute_integrals`` stores in ``IntegralSet.ERI``
instead of the dense (n,n,n,n) tensor of ``jax_qc/integrals/eri.py:69-105``,
and what the Fock builders contract against.

All matrices are torch float64 tensors on the engine's CUDA device.  Spherical
basis sets (the reference default, ``basis/build.py:28``) are handled by the
N^2 transform C (``spherical.py:34-67``): D_cart = C^T D C, J = C J_cart C^T.
"""

from __future__ import annotations

import ctypes
import math
from typing import Optional, Tuple

import numpy as np
import torch

from . import _abi
from .core import n_cartesian


def _require_cuda(device) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError(
            "jax_examples_b200 needs a CUDA device: the two-electron path runs only in libjqc.so "
            "(no CPU fallback)"
        )
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else int(device))
    return dev


def _stream(dev: torch.device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def cart_to_spherical(l: int) -> np.ndarray:
    """(2l+1, ncart(l)) real-solid-harmonic map in libcint row order, the
    same table as ``jax_qc/integrals/spherical.py:34-67`` (l <= 2)."""
    if l == 0:
        return np.array([[1.0]])
    if l == 1:
        return np.eye(3)
    if l == 2:
        r3 = math.sqrt(3.0)
        return np.array(
            [
                [0.0, r3, 0.0, 0.0, 0.0, 0.0],
                [0.0, 0.0, 0.0, 0.0, r3, 0.0],
                [-0.5, 0.0, 0.0, -0.5, 0.0, 1.0],
                [0.0, 0.0, r3, 0.0, 0.0, 0.0],
                [r3 / 2.0, 0.0, 0.0, -r3 / 2.0, 0.0, 0.0],
            ]
        )
    raise NotImplementedError(
        f"Cart-to-spherical transformation only implemented for l <= 2 (got l={l})."
    )


class PackedBasis:
    """SoA view of any reference-style basis (``.shells`` of Shell records)."""

    def __init__(self, basis):
        shells = basis.shells
        self.n_shell = len(shells)
        self.l = np.array([int(s.angular_momentum) for s in shells], dtype=np.int32)
        self.nprim = np.array([len(np.asarray(s.exponents)) for s in shells], dtype=np.int32)
        self.prim_off = np.concatenate([[0], np.cumsum(self.nprim)[:-1]]).astype(np.int32)
        self.exps = np.ascontiguousarray(np.concatenate([np.asarray(s.exponents, np.float64) for s in shells]))
        self.coefs = np.ascontiguousarray(np.concatenate([np.asarray(s.coefficients, np.float64) for s in shells]))
        self.centres = np.ascontiguousarray(np.array([np.asarray(s.center, np.float64) for s in shells]))
        self.atom = np.array([int(s.atom_index) for s in shells], dtype=np.int32)
        self.n_cart = int(sum(n_cartesian(int(x)) for x in self.l))
        self.spherical = bool(getattr(basis, "spherical", False))
        self.n_basis = int(sum((2 * int(x) + 1) if self.spherical else n_cartesian(int(x)) for x in self.l))


class DirectERI:
    """Direct (integral-direct) two-electron engine for one basis/geometry.

    Args:
        basis: BasisSet (this package's or the reference's).
        mol: Molecule providing nuclei for the one-electron and gradient
            kernels; optional for pure two-electron use.
        device: CUDA device index (default: current).
        schwarz_tau: shell quartets with Q_ij Q_kl below this are skipped.
        prim_tau: primitive pairs of magnitude below this are dropped
            (1e-20 changes no integral by more than ~1e-19).
        mol_of_atom: optional molecule index of every atom when the basis
            and nuclei are a batch of independent molecules
            (``jqc_batch_partition``); matrices are then the block-diagonal
            matrices of the whole batch.
    """

    def __init__(self, basis, mol=None, device=None, schwarz_tau: float = 1e-13, prim_tau: float = 1e-20,
                 mol_of_atom=None):
        self.device = _require_cuda(device)
        self.lib = _abi.load()
        self.basis = basis
        self.packed = pk = PackedBasis(basis)
        self.schwarz_tau = float(schwarz_tau)
        self.prim_tau = float(prim_tau)
        if mol is not None:
            self.atom_xyz = np.ascontiguousarray(np.asarray(mol.coords, np.float64))
            self.atom_Z = np.ascontiguousarray(np.asarray(mol.atomic_numbers, np.float64))
        else:
            n_atom = int(pk.atom.max()) + 1
            self.atom_xyz = np.zeros((n_atom, 3))
            for s in range(pk.n_shell):
                self.atom_xyz[pk.atom[s]] = pk.centres[s]
            self.atom_Z = np.zeros(n_atom)
        self._ctx = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _abi.call("jqc_ctx_create", self.device.index, ctypes.byref(self._ctx))
            ip = lambda a: a.ctypes.data_as(_abi._ip)  # noqa: E731
            dp = lambda a: a.ctypes.data_as(_abi._dp)  # noqa: E731
            _abi.call(
                "jqc_basis_upload", self._ctx, pk.n_shell, ip(pk.l), ip(pk.nprim), ip(pk.prim_off), dp(pk.exps),
                dp(pk.coefs), dp(pk.centres), ip(pk.atom), len(self.atom_Z), dp(self.atom_xyz), dp(self.atom_Z), 1,
            )
            self.n_mol = 1
            if mol_of_atom is not None:
                moa = np.ascontiguousarray(np.asarray(mol_of_atom, dtype=np.int32))
                if moa.shape != (len(self.atom_Z),):
                    raise ValueError(f"mol_of_atom must have one entry per atom ({len(self.atom_Z)})")
                self.n_mol = int(moa.max()) + 1 if moa.size else 1
                _abi.call("jqc_batch_partition", self._ctx, self.n_mol, ip(moa))
            _abi.call("jqc_pairs_build", self._ctx, self.schwarz_tau, float(prim_tau), _stream(self.device))
        self._C = None
        if pk.spherical:
            C = np.zeros((pk.n_basis, pk.n_cart))
            r = c = 0
            for l in pk.l:
                m = cart_to_spherical(int(l))
                C[r:r + m.shape[0], c:c + m.shape[1]] = m
                r += m.shape[0]
                c += m.shape[1]
            self._C = torch.tensor(C, dtype=torch.float64, device=self.device)

    # ------------------------------------------------------------ geometry
    def set_geometry(self, coords, active=None) -> None:
        """Move the nuclei (and every shell with its atom) to ``coords``
        (n_atom, 3) bohr and rebuild the shell pairs, keeping the basis, the
        batch partition and the launch tuning (``jqc_set_geometry`` +
        ``jqc_pairs_build``).  ``active`` (one flag per molecule of the batch
        partition) leaves the pairs of inactive molecules out of the builds."""
        xyz = np.ascontiguousarray(np.asarray(coords, dtype=np.float64))
        if xyz.shape != self.atom_xyz.shape:
            raise ValueError(f"coords must have shape {self.atom_xyz.shape}; got {xyz.shape}")
        dp = lambda a: a.ctypes.data_as(_abi._dp)  # noqa: E731
        with torch.cuda.device(self.device):
            _abi.call("jqc_set_geometry", self._ctx, dp(xyz))
            if active is not None:
                act = np.ascontiguousarray(np.asarray(active, dtype=np.int32))
                if act.shape != (self.n_mol,):
                    raise ValueError(f"active must have one flag per molecule ({self.n_mol})")
                _abi.call("jqc_set_molecule_mask", self._ctx, act.ctypes.data_as(_abi._ip))
            else:
                _abi.call("jqc_set_molecule_mask", self._ctx, None)
            _abi.call("jqc_pairs_build", self._ctx, self.schwarz_tau, float(self.prim_tau), _stream(self.device))
        self.atom_xyz = xyz
        self.packed.centres = np.ascontiguousarray(xyz[self.packed.atom])

    def set_molecule_activity(self, flags: Optional[torch.Tensor]) -> None:
        """Device flags (int32, one per molecule of the batch partition) that
        every later J/K build reads on the device: molecules flagged 0 are
        compacted out of the work before the class kernels run
        (``jqc_set_molecule_activity``).  ``None`` switches it off.  The
        engine keeps a reference to the tensor; rewrite it in place."""
        if flags is not None:
            if not (flags.is_cuda and flags.dtype == torch.int32 and flags.is_contiguous()
                    and flags.numel() == self.n_mol and flags.device == self.device):
                raise ValueError(f"flags must be a contiguous int32 tensor of {self.n_mol} entries on {self.device}")
        with torch.cuda.device(self.device):
            _abi.call("jqc_set_molecule_activity", self._ctx, None if flags is None else _ptr(flags))
        self._activity = flags

    # ------------------------------------------------------------ lifecycle
    def close(self) -> None:
        if getattr(self, "_ctx", None) is not None and self._ctx.value:
            try:
                self.lib.jqc_ctx_destroy(self._ctx)
            finally:
                self._ctx = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_basis(self) -> int:
        return self.packed.n_basis

    @property
    def shape(self):
        n = self.n_basis
        return (n, n, n, n)

    # ------------------------------------------------------------- helpers
    def _to_cart(self, D: torch.Tensor) -> torch.Tensor:
        return D if self._C is None else self._C.T @ D @ self._C

    def _from_cart(self, M: torch.Tensor) -> torch.Tensor:
        return M if self._C is None else self._C @ M @ self._C.T

    def _dens(self, D) -> Tuple[torch.Tensor, bool]:
        D = torch.as_tensor(D, dtype=torch.float64, device=self.device)
        single = D.dim() == 2
        if single:
            D = D[None]
        n = self.n_basis
        if D.dim() != 3 or D.shape[1:] != (n, n):
            raise ValueError(f"density must be ({n},{n}) or (k,{n},{n}); got {tuple(D.shape)}")
        return D, single

    # ----------------------------------------------------------------- API
    def jk(self, D, precision: str = "fp64", mixed_tau: float = 1e-7, dens_tau: float = 0.0):
        """J and K for one density (n,n) or a stack (k,n,n), k <= 4."""
        if precision not in _abi.PREC:
            raise ValueError(f"precision must be one of {sorted(_abi.PREC)}")
        D, single = self._dens(D)
        if self._C is not None:
            D = torch.stack([self._to_cart(d) for d in D])
        D = D.contiguous()
        k, nc = D.shape[0], self.packed.n_cart
        J = torch.empty((k, nc, nc), dtype=torch.float64, device=self.device)
        K = torch.empty_like(J)
        with torch.cuda.device(self.device):
            _abi.call("jqc_jk", self._ctx, k, _ptr(D), _ptr(J), _ptr(K), _abi.PREC[precision], float(mixed_tau),
                      float(dens_tau), _stream(self.device))
        if self._C is not None:
            J = torch.stack([self._from_cart(m) for m in J])
            K = torch.stack([self._from_cart(m) for m in K])
        return (J[0], K[0]) if single else (J, K)

    def eri_tensor(self, max_bytes: int = 32 << 30) -> torch.Tensor:
        """Dense (n,n,n,n) tensor, for small systems and parity checks."""
        nc = self.packed.n_cart
        if nc ** 4 * 8 > max_bytes:
            raise _abi.JQCTooLarge(f"n^4 tensor of {nc ** 4 * 8 / 2 ** 30:.1f} GiB exceeds max_bytes")
        out = torch.empty((nc,) * 4, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _abi.call("jqc_eri_tensor", self._ctx, _ptr(out), int(max_bytes), _stream(self.device))
        if self._C is not None:
            # one index at a time (a single four-operand einsum may contract
            # the C factors with each other first, an n^8 intermediate)
            C = self._C
            out = torch.tensordot(C, out, dims=([1], [0]))
            out = torch.tensordot(C, out, dims=([1], [1])).transpose(0, 1)
            out = torch.tensordot(out, C, dims=([2], [1])).transpose(2, 3)
            out = torch.tensordot(out, C, dims=([3], [1])).contiguous()
        return out

    def one_electron(self):
        """(S, T, V) in the engine's basis layout."""
        nc = self.packed.n_cart
        S, T, V = (torch.empty((nc, nc), dtype=torch.float64, device=self.device) for _ in range(3))
        with torch.cuda.device(self.device):
            _abi.call("jqc_one_electron", self._ctx, _ptr(S), _ptr(T), _ptr(V), _stream(self.device))
        return self._from_cart(S), self._from_cart(T), self._from_cart(V)

    def schwarz(self) -> torch.Tensor:
        ns = self.packed.n_shell
        Q = torch.empty((ns, ns), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _abi.call("jqc_schwarz", self._ctx, _ptr(Q), _stream(self.device))
        return Q

    def jk_timed(self, D, precision: str = "fp64", mixed_tau: float = 1e-7, dens_tau: float = 0.0):
        """J/K with the class kernels serialized and timed; returns
        (J, K, ms) with ms[(p*21+q)] per class (measurement helper)."""
        D, single = self._dens(D)
        if self._C is not None:
            D = torch.stack([self._to_cart(d) for d in D])
        D = D.contiguous()
        k, nc = D.shape[0], self.packed.n_cart
        J = torch.empty((k, nc, nc), dtype=torch.float64, device=self.device)
        K = torch.empty_like(J)
        ms = (ctypes.c_double * 42)()
        with torch.cuda.device(self.device):
            _abi.call("jqc_jk_timed", self._ctx, k, _ptr(D), _ptr(J), _ptr(K), _abi.PREC[precision],
                      float(mixed_tau), float(dens_tau), _stream(self.device), ms)
        return J, K, list(ms)

    def class_stats(self, precision: str = "fp64", mixed_tau: float = 1e-7):
        """[(path, class_index, quartets, prim_quartets, tasks)] for non-empty classes."""
        out = (ctypes.c_longlong * 126)()
        with torch.cuda.device(self.device):
            _abi.call("jqc_class_stats", self._ctx, _abi.PREC[precision], float(mixed_tau), out)
        rows = []
        for p in range(2):
            for q in range(21):
                k = (p * 21 + q) * 3
                if out[k]:
                    rows.append((p, q, out[k], out[k + 1], out[k + 2]))
        return rows

    def stats(self, precision: str = "fp64", mixed_tau: float = 1e-7) -> dict:
        out = (ctypes.c_longlong * 8)()
        with torch.cuda.device(self.device):
            _abi.call("jqc_stats", self._ctx, _abi.PREC[precision], float(mixed_tau), out)
        return {
            "shell_pairs": out[0],
            "kept_pairs": out[1],
            "quartets_fp64": out[2],
            "quartets_fp32": out[3],
            "prim_quartets": out[4],
            "n_cart": out[5],
            "tasks": out[6],
            "launches_per_jk": out[7],
        }


# Quartet class q -> (la, lb, lc, ld), bra pair class >= ket pair class.
PAIR_CLASSES = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]
QUARTET_CLASSES = [PAIR_CLASSES[pb] + PAIR_CLASSES[pk] for pb in range(6) for pk in range(pb + 1)]


def fp_peak(fp32: bool = False, blocks: int = 148 * 8, iters: int = 4096) -> float:
    """Measured FMA throughput of the current device in TFLOP/s."""
    out = ctypes.c_double()
    _abi.call("jqc_fp_peak", int(bool(fp32)), int(blocks), int(iters), ctypes.byref(out),
              _stream(torch.device("cuda", torch.cuda.current_device())))
    return out.value


def boys(T: torch.Tensor, mmax: int, fp32: bool = False) -> torch.Tensor:
    """F_m(T), m = 0..mmax, on the device (``jqc_boys``)."""
    T = torch.as_tensor(T, dtype=torch.float64).contiguous()
    if not T.is_cuda:
        raise ValueError("T must be a CUDA tensor")
    out = torch.empty((T.numel(), mmax + 1), dtype=torch.float32 if fp32 else torch.float64, device=T.device)
    with torch.cuda.device(T.device):
        _abi.call("jqc_boys", _ptr(T), T.numel(), int(mmax), _ptr(out), int(bool(fp32)), _stream(T.device))
    return out


def eri_prim_quartets(cls, exps: torch.Tensor, centres: torch.Tensor) -> torch.Tensor:
    """Primitive Cartesian blocks for quartets of one class (``jqc_eri_prim_quartets``).

    ``exps`` (n,4) and ``centres`` (n,4,3) float64 CUDA tensors; returns
    (n, nc_a, nc_b, nc_c, nc_d)."""
    la, lb, lc, ld = (int(x) for x in cls)
    exps = torch.as_tensor(exps, dtype=torch.float64).contiguous()
    centres = torch.as_tensor(centres, dtype=torch.float64).contiguous()
    n = exps.shape[0]
    shp = (n, n_cartesian(la), n_cartesian(lb), n_cartesian(lc), n_cartesian(ld))
    out = torch.empty(shp, dtype=torch.float64, device=exps.device)
    with torch.cuda.device(exps.device):
        _abi.call("jqc_eri_prim_quartets", la, lb, lc, ld, n, _ptr(exps), _ptr(centres), _ptr(out),
                  _stream(exps.device))
    return out
