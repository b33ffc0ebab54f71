"""TEST INFRASTRUCTURE ONLY -- CPU oracle of the jax_qc two-electron path.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker / the timed CPU port.
The product package ``jax_examples_b200`` never imports it.

The arithmetic lives in ``mmd_oracle.c`` (a C restatement of the reference's
``boys.py``, ``mcmurchie_davidson.py``, ``obara_saika.py``, ``eri.py``,
``screening.py`` and ``fock.py``); this module adds ctypes bindings and NumPy
restatements of the reference's host-side drivers:

* ``rhf`` / ``uhf``: ``jax_qc/scf/rhf.py:95-169``, ``scf/uhf.py:187-287`` with
  ``scf/diis.py:53-199``, ``guess.py:25-115``, ``density.py``, ``energy.py``.
* ``rhf_gradient_fd``: ``jax_qc/grad/rhf_grad.py:106-211`` (central finite
  differences of S, H and the ERI tensor at fixed density).
* ``numerical_gradient``: ``jax_qc/grad/numerical_grad.py:51-94``.

``mode`` selects the Boys function: 0 = the reference's as-is ``boys_fn``
(inaccurate for n>=3 at small t), 1 = accurate.  Parity of this oracle with
the reference itself is pinned by ``tests/golden`` (fixtures made by running
the reference's own code).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Callable, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build() -> str:
    """Compile ``liboracle.so`` (gcc, OpenMP) if it is missing or stale."""
    so = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "mmd_oracle.c")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return so


def lib():
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(build())
        _LIB.oracle_boys_ref.restype = ctypes.c_double
        _LIB.oracle_boys_ref.argtypes = [ctypes.c_int, ctypes.c_double]
        _LIB.oracle_boys_exact.restype = ctypes.c_double
        _LIB.oracle_boys_exact.argtypes = [ctypes.c_int, ctypes.c_double]
    return _LIB


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_dp)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32).ctypes.data_as(_ip)


# --------------------------------------------------------------------- Boys


def boys_ref(n: int, t: float) -> float:
    return lib().oracle_boys_ref(int(n), float(t))


def boys_exact(n: int, t: float) -> float:
    return lib().oracle_boys_exact(int(n), float(t))


def boys_array(T, mmax: int, mode: int = 1) -> np.ndarray:
    """F_m(T) for m = 0..mmax, shape (len(T), mmax+1)."""
    T = np.ascontiguousarray(T, dtype=np.float64)
    out = np.empty((T.size, mmax + 1), dtype=np.float64)
    lib().oracle_boys_array(ctypes.c_int(mode), _d(T), ctypes.c_longlong(T.size), ctypes.c_int(mmax),
                            out.ctypes.data_as(_dp))
    return out


# ------------------------------------------------------------ MMD kernels


def hermite_e(la, lb, xpa, xpb, p) -> np.ndarray:
    out = np.empty((la + 1, lb + 1, la + lb + 1))
    lib().oracle_hermite_e(ctypes.c_int(la), ctypes.c_int(lb), ctypes.c_double(xpa), ctypes.c_double(xpb),
                           ctypes.c_double(p), out.ctypes.data_as(_dp))
    return out


def hermite_r(tmax, umax, vmax, p, PC, mode: int = 1) -> np.ndarray:
    out = np.empty((tmax + 1, umax + 1, vmax + 1))
    lib().oracle_hermite_r(ctypes.c_int(tmax), ctypes.c_int(umax), ctypes.c_int(vmax), ctypes.c_double(p),
                           _d(np.asarray(PC, dtype=np.float64)), ctypes.c_int(mode), out.ctypes.data_as(_dp))
    return out


def _nc(l):
    return (l + 1) * (l + 2) // 2


def primitive_eri(alpha, A, la, beta, B, lb, gamma, C, lc, delta, D, ld, mode: int = 1) -> np.ndarray:
    out = np.empty((_nc(la), _nc(lb), _nc(lc), _nc(ld)))
    A, B, C, D = (np.ascontiguousarray(x, dtype=np.float64) for x in (A, B, C, D))
    lib().oracle_primitive_eri(
        ctypes.c_double(alpha), A.ctypes.data_as(_dp), ctypes.c_int(la),
        ctypes.c_double(beta), B.ctypes.data_as(_dp), ctypes.c_int(lb),
        ctypes.c_double(gamma), C.ctypes.data_as(_dp), ctypes.c_int(lc),
        ctypes.c_double(delta), D.ctypes.data_as(_dp), ctypes.c_int(ld),
        ctypes.c_int(mode), out.ctypes.data_as(_dp))
    return out


class Packed:
    """SoA view of a basis (any object with ``.shells`` of reference-style
    Shell records)."""

    def __init__(self, basis):
        shells = basis.shells
        self.n_shell = len(shells)
        self.l = np.array([int(s.angular_momentum) for s in shells], dtype=np.int32)
        self.nprim = np.array([len(np.asarray(s.exponents)) for s in shells], dtype=np.int32)
        self.prim_off = np.concatenate([[0], np.cumsum(self.nprim)[:-1]]).astype(np.int32)
        self.exps = np.concatenate([np.asarray(s.exponents, dtype=np.float64) for s in shells])
        self.coefs = np.concatenate([np.asarray(s.coefficients, dtype=np.float64) for s in shells])
        self.centres = np.ascontiguousarray(np.array([np.asarray(s.center, dtype=np.float64) for s in shells]))
        self.atom = np.array([int(s.atom_index) for s in shells], dtype=np.int32)
        self.n = int(sum(_nc(int(x)) for x in self.l))
        self.offsets = np.concatenate([[0], np.cumsum([_nc(int(x)) for x in self.l])]).astype(np.int64)

    def args(self):
        return (ctypes.c_int(self.n_shell), _i(self.l), _i(self.nprim), _i(self.prim_off), _d(self.exps),
                _d(self.coefs), _d(self.centres))


def contracted_eri(basis, I, J, K, L, mode: int = 1) -> np.ndarray:
    pk = basis if isinstance(basis, Packed) else Packed(basis)
    l = pk.l
    out = np.empty((_nc(l[I]), _nc(l[J]), _nc(l[K]), _nc(l[L])))
    lib().oracle_contracted_eri(*pk.args(), ctypes.c_int(I), ctypes.c_int(J), ctypes.c_int(K), ctypes.c_int(L),
                                ctypes.c_int(mode), out.ctypes.data_as(_dp))
    return out


def eri_tensor(basis, mode: int = 1) -> np.ndarray:
    """Dense Cartesian (n,n,n,n) tensor exactly as ``eri.py:69-105`` builds it."""
    pk = basis if isinstance(basis, Packed) else Packed(basis)
    out = np.zeros((pk.n,) * 4)
    lib().oracle_eri_tensor(*pk.args(), ctypes.c_int(mode), ctypes.c_int(pk.n), out.ctypes.data_as(_dp))
    return out


def schwarz(basis, mode: int = 1) -> np.ndarray:
    """Q[i,j] = sqrt(max (ij|ij)) (``screening.py:32-58``)."""
    pk = basis if isinstance(basis, Packed) else Packed(basis)
    out = np.zeros((pk.n_shell, pk.n_shell))
    lib().oracle_schwarz(*pk.args(), ctypes.c_int(mode), out.ctypes.data_as(_dp))
    return out


def jk_from_tensor(D, eri):
    """``fock.py:31-38``: J = einsum('ls,mnls'), K = einsum('ls,msln')."""
    n = D.shape[0]
    J = np.empty((n, n))
    K = np.empty((n, n))
    lib().oracle_jk_from_tensor(ctypes.c_int(n), _d(D), _d(eri), J.ctypes.data_as(_dp), K.ctypes.data_as(_dp))
    return J, K


def canonical_quartets(n_shell: int) -> np.ndarray:
    """All (i, j, k, l) with i>=j, k>=l, ij>=kl in the reference's loop order
    (``eri.py:89-96``)."""
    out = []
    for i in range(n_shell):
        for j in range(i + 1):
            ij = i * (i + 1) // 2 + j
            for k in range(n_shell):
                for l in range(k + 1):
                    if ij >= k * (k + 1) // 2 + l:
                        out.append((i, j, k, l))
    return np.array(out, dtype=np.int32).reshape(-1, 4)


def jk_quartets(basis, D, quartets=None, mode: int = 1):
    """J/K digested directly from a list of canonical shell quartets (no dense
    tensor).  Over the full canonical list this equals ``jk_from_tensor``."""
    pk = basis if isinstance(basis, Packed) else Packed(basis)
    if quartets is None:
        quartets = canonical_quartets(pk.n_shell)
    q = np.ascontiguousarray(quartets, dtype=np.int32)
    J = np.empty((pk.n, pk.n))
    K = np.empty((pk.n, pk.n))
    lib().oracle_jk_quartets(*pk.args(), ctypes.c_int(mode), ctypes.c_int(pk.n), ctypes.c_longlong(len(q)),
                             _i(q), _d(D), J.ctypes.data_as(_dp), K.ctypes.data_as(_dp))
    return J, K


def one_electron(basis, mol, mode: int = 1):
    """S, T, V (Cartesian) as ``overlap.py``/``kinetic.py``/``nuclear.py`` build them."""
    pk = basis if isinstance(basis, Packed) else Packed(basis)
    xyz = np.ascontiguousarray(np.asarray(mol.coords, dtype=np.float64))
    Z = np.ascontiguousarray(np.asarray(mol.atomic_numbers, dtype=np.float64))
    S, T, V = (np.zeros((pk.n, pk.n)) for _ in range(3))
    lib().oracle_one_electron(*pk.args(), ctypes.c_int(len(Z)), _d(xyz), _d(Z), ctypes.c_int(mode),
                              ctypes.c_int(pk.n), S.ctypes.data_as(_dp), T.ctypes.data_as(_dp),
                              V.ctypes.data_as(_dp))
    return S, T, V


def nuclear_repulsion(coords, Z) -> float:
    """``nuclear.py:84-98`` / ``rhf_grad.py:214-222``."""
    coords = np.asarray(coords, dtype=np.float64)
    Z = np.asarray(Z, dtype=np.float64)
    total = 0.0
    for i in range(len(Z)):
        for j in range(i + 1, len(Z)):
            total += Z[i] * Z[j] / float(np.linalg.norm(coords[i] - coords[j]))
    return total


# ---------------------------------------------------------------- spherical


def cart_to_spherical(l: int) -> np.ndarray:
    """(2l+1, ncart) map of ``integrals/spherical.py:34-67``: identity for
    s and p; for d the real solid harmonics in libcint row order
    (xy, yz, z^2, xz, x^2-y^2) over the Cartesian columns xx, xy, xz, yy,
    yz, zz, all components sharing one normalization."""
    if l == 0:
        return np.ones((1, 1))
    if l == 1:
        return np.eye(3)
    if l == 2:
        m = np.zeros((5, 6))
        r3 = np.sqrt(3.0)
        m[0, 1] = r3
        m[1, 4] = r3
        m[2, [0, 3, 5]] = (-0.5, -0.5, 1.0)
        m[3, 2] = r3
        m[4, [0, 3]] = (r3 / 2.0, -r3 / 2.0)
        return m
    raise NotImplementedError(f"Cart-to-spherical transformation only implemented for l <= 2 (got l={l}).")


def spherical_matrix(basis) -> np.ndarray:
    """Block-diagonal C (n_sph, n_cart) over the shells in basis order, so
    that M_sph = C M_cart C^T (``eri.py:61-66,100-103`` per block)."""
    blocks = [cart_to_spherical(int(s.angular_momentum)) for s in basis.shells]
    C = np.zeros((sum(b.shape[0] for b in blocks), sum(b.shape[1] for b in blocks)))
    r = c = 0
    for b in blocks:
        C[r:r + b.shape[0], c:c + b.shape[1]] = b
        r += b.shape[0]
        c += b.shape[1]
    return C


def eri_to_spherical(eri, C) -> np.ndarray:
    """(pq|rs) = sum C_pi C_qj C_rk C_sl (ij|kl), one index at a time."""
    t = np.tensordot(C, eri, axes=(1, 0))
    t = np.tensordot(C, t, axes=(1, 1)).transpose(1, 0, 2, 3)
    t = np.tensordot(t, C, axes=(2, 1)).transpose(0, 1, 3, 2)
    return np.tensordot(t, C, axes=(3, 1))


# ---------------------------------------------------------------- SCF / DIIS


def _sym_orth(S):
    w, U = np.linalg.eigh(S)
    return U @ np.diag(1.0 / np.sqrt(w)) @ U.T


def _diag(F, X):
    e, Cp = np.linalg.eigh(X.T @ F @ X)
    return e, X @ Cp


def _diis_error(F, D, S, X):
    return X.T @ (F @ D @ S - S @ D @ F) @ X


def _diis_solve(errors):
    m = len(errors)
    B = np.empty((m + 1, m + 1))
    for i in range(m):
        for j in range(m):
            B[i, j] = float(np.sum(errors[i] * errors[j]))
    B[-1, :-1] = -1.0
    B[:-1, -1] = -1.0
    B[-1, -1] = 0.0
    rhs = np.zeros(m + 1)
    rhs[-1] = -1.0
    try:
        return np.linalg.solve(B, rhs)[:-1]
    except np.linalg.LinAlgError:
        return None


class _DIIS:
    """Ring buffer of ``diis.py:26-130``: evict oldest when full."""

    def __init__(self, size):
        self.size = size
        self.F, self.E = [], []

    def extrapolate(self, F, e):
        self.F.append(F)
        self.E.append(e)
        if len(self.F) > self.size:
            self.F.pop(0)
            self.E.pop(0)
        if len(self.F) < 2:
            return F
        c = _diis_solve(self.E)
        if c is None:
            return F
        return np.einsum("i,imn->mn", c, np.array(self.F))


def rhf(S, H, jk: Callable, n_occ: int, conv: float = 1e-10, max_iter: int = 128, diis_space: int = 8,
        damping: float = 0.0):
    """``rhf.py:95-169``; ``jk(D) -> (J, K)``.  Returns (E_elec, D, C, eps, F, n_iter, converged)."""
    X = _sym_orth(S)
    _, C = _diag(H, X)
    D = 2.0 * C[:, :n_occ] @ C[:, :n_occ].T
    J, K = jk(D)
    F = H + J - 0.5 * K
    eps, C = _diag(F, X)
    E = 0.5 * np.sum(D * (H + F))
    diis = _DIIS(diis_space)
    last, conv_ok, it = E, False, 0
    for it in range(1, max_iter + 1):
        J, K = jk(D)
        Fn = H + J - 0.5 * K
        if damping > 0:
            Fn = (1 - damping) * Fn + damping * F
        err = _diis_error(Fn, D, S, X)
        F = diis.extrapolate(Fn, err)
        eps, C = _diag(F, X)
        D = 2.0 * C[:, :n_occ] @ C[:, :n_occ].T
        E = 0.5 * np.sum(D * (H + F))
        dE = abs(E - last)
        last = E
        if dE < conv and np.max(np.abs(err)) < max(conv, 1e-6):
            conv_ok = True
            break
    return E, D, C, eps, F, it, conv_ok


def uhf(S, H, jk: Callable, n_alpha: int, n_beta: int, conv: float = 1e-10, max_iter: int = 128,
        diis_space: int = 8, damping: float = 0.0):
    """``uhf.py:187-287`` with the alpha-repulsion guess of ``guess.py:42-115``.
    ``jk(D) -> (J, K)``.  Returns (E_elec, Da, Db, n_iter, converged)."""
    X = _sym_orth(S)
    n = S.shape[0]
    _, Ca = _diag(H, X)
    if n_alpha != n_beta:
        Dai = Ca[:, :n_alpha] @ Ca[:, :n_alpha].T
        Ja, Ka = jk(Dai)
        Fb = H + Ja - Ka
        ev = np.linalg.eigvalsh(X.T @ Fb @ X)
        scale = 0.01 * float(ev.max() - ev.min()) + 0.1
        idx = np.arange(n, dtype=np.float64)
        noise = scale * np.outer(np.sin(idx * 1.23 + 0.45), np.cos(idx * 0.67 + 0.89))
        Fb = Fb + (noise + noise.T) / 2.0
        _, Cb = _diag(Fb, X)
    else:
        Cb = Ca
    Da = Ca[:, :n_alpha] @ Ca[:, :n_alpha].T
    Db = Cb[:, :n_beta] @ Cb[:, :n_beta].T

    def fock(Da, Db):
        Ja, Ka = jk(Da)
        Jb, Kb = jk(Db)
        return H + Ja + Jb - Ka, H + Ja + Jb - Kb

    Fa, Fb = fock(Da, Db)
    _, Ca = _diag(Fa, X)
    _, Cb = _diag(Fb, X)
    Da = Ca[:, :n_alpha] @ Ca[:, :n_alpha].T
    Db = Cb[:, :n_beta] @ Cb[:, :n_beta].T
    E = 0.5 * np.sum(Da * (H + Fa)) + 0.5 * np.sum(Db * (H + Fb))
    diis = _DIIS(diis_space)
    last, ok, it = E, False, 0
    init_damp = 0.3 if n_alpha != n_beta else 0.0
    for it in range(max_iter):
        dmp = init_damp if it < 5 else damping
        Fan, Fbn = fock(Da, Db)
        if dmp > 0:
            Fan = (1 - dmp) * Fan + dmp * Fa
            Fbn = (1 - dmp) * Fbn + dmp * Fb
        ea = _diis_error(Fan, Da, S, X)
        eb = _diis_error(Fbn, Db, S, X)
        Fc = diis.extrapolate(np.concatenate([Fan, Fbn]), np.concatenate([ea, eb]))
        Fa, Fb = Fc[:n], Fc[n:]
        _, Ca = _diag(Fa, X)
        _, Cb = _diag(Fb, X)
        Da = Ca[:, :n_alpha] @ Ca[:, :n_alpha].T
        Db = Cb[:, :n_beta] @ Cb[:, :n_beta].T
        E = 0.5 * np.sum(Da * (H + Fa)) + 0.5 * np.sum(Db * (H + Fb))
        err = max(np.max(np.abs(ea)), np.max(np.abs(eb)))
        dE = abs(E - last)
        last = E
        if dE < conv and err < max(conv, 1e-6):
            ok = True
            break
    return E, Da, Db, it + 1, ok


# ------------------------------------------------------------ gradients


def rhf_energy(mol, build_basis: Callable, mode: int = 1, conv: float = 1e-10, spherical: bool = False):
    """Total RHF energy through the oracle (dense tensor; small systems).
    ``spherical`` runs the SCF in the solid-harmonic basis of the shells, as
    the reference does for ``BasisSet.spherical``."""
    basis = build_basis(mol)
    S, T, V = one_electron(basis, mol, mode)
    eri = eri_tensor(basis, mode)
    if spherical:
        C = spherical_matrix(basis)
        S, T, V = (C @ M @ C.T for M in (S, T, V))
        eri = eri_to_spherical(eri, C)
    E, D, C, eps, F, it, ok = rhf(S, T + V, lambda D: jk_from_tensor(D, eri), mol.n_electrons // 2, conv=conv)
    return E + nuclear_repulsion(mol.coords, mol.atomic_numbers), D, C, eps, ok


def rhf_gradient_fd(mol, build_basis: Callable, D, C, eps, step: float = 1e-4, mode: int = 1,
                    displace: Optional[Callable] = None):
    """``rhf_grad.py:106-211``: integral derivatives by central differences at
    fixed D and W; ``displace(mol, coords)`` builds the displaced molecule."""
    coords = np.asarray(mol.coords, dtype=np.float64)
    Z = np.asarray(mol.atomic_numbers, dtype=np.float64)
    n_occ = mol.n_electrons // 2
    W = 2.0 * (C[:, :n_occ] * eps[:n_occ][None, :]) @ C[:, :n_occ].T
    g = np.zeros_like(coords)
    for a in range(len(Z)):
        for k in range(3):
            cp, cm = coords.copy(), coords.copy()
            cp[a, k] += step
            cm[a, k] -= step
            mp, mm = displace(mol, cp), displace(mol, cm)
            bp, bm = build_basis(mp), build_basis(mm)
            Sp, Tp, Vp = one_electron(bp, mp, mode)
            Sm, Tm, Vm = one_electron(bm, mm, mode)
            Ep, Em = eri_tensor(bp, mode), eri_tensor(bm, mode)
            dH = ((Tp + Vp) - (Tm + Vm)) / (2 * step)
            dS = (Sp - Sm) / (2 * step)
            dERI = (Ep - Em) / (2 * step)
            dJ, dK = jk_from_tensor(D, dERI)
            dEn = (nuclear_repulsion(cp, Z) - nuclear_repulsion(cm, Z)) / (2 * step)
            g[a, k] = dEn + np.sum(D * dH) + 0.5 * np.sum(D * (dJ - 0.5 * dK)) - np.sum(W * dS)
    return g
