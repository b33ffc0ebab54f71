"""Basis construction: BSE-schema dicts -> normalized contracted shells.

Follows the reference's basis layer:

* ``primitive_norm`` / ``contraction_norm`` / ``normalize_shell`` restate
  ``jax_qc/basis/normalize.py:36-107`` (one N_l per shell, shared by every
  Cartesian component).
* ``bse_dict_to_shells`` restates ``jax_qc/basis/parse.py:26-127``: one shell
  per (l, contraction row), zero coefficients dropped, per-atom sort by
  (l ascending, largest exponent descending).
* ``build_shell_indices`` restates ``jax_qc/basis/parse.py:130-152``.

Basis data.  The Basis Set Exchange database is not available, so the named
bases here are:

* ``"sto-3g"`` (H, He, C, N, O, F), ``"6-31g"``, ``"6-31g*"`` and
  ``"6-31g**"`` (H, O): the published parameters, carried as constant tables
  in :mod:`.basis_data` (He STO-3G is the reference's own table,
  ``fp/qchem_fp.py:64-76``).
* ``"syn-sto-3g"``, ``"syn-6-31g*"``, ``"syn-6-31g**"``: *synthetic* bases
  with the shell structure and contraction lengths of STO-3G / 6-31G* /
  6-31G** (Cartesian d) and exponents/coefficients generated from simple
  closed-form sequences.  They exercise the kernels with other exponent
  spreads; no workload of the benchmark uses them.

Any real basis can be used by passing its BSE-schema dict to
:func:`build_basis_set` (``basis=dict``) or by registering it with
:func:`register_basis`.
"""

from __future__ import annotations

import math
from typing import Dict, List

import numpy as np

from .basis_data import real_bases
from .core import (
    ANGSTROM_TO_BOHR,
    BasisSet,
    Molecule,
    Shell,
    make_molecule,
    n_cartesian,
)


# ---------------------------------------------------------------------------
# normalization (jax_qc/basis/normalize.py)
# ---------------------------------------------------------------------------


def double_factorial(n: int) -> int:
    """n!! with (-1)!! = 0!! = 1 (``normalize.py:20-33``)."""
    result = 1
    k = n
    while k > 1:
        result *= k
        k -= 2
    return result


def primitive_norm(alpha: float, l: int) -> float:
    """(2a/pi)^(3/4) sqrt((4a)^l / (2l-1)!!) (``normalize.py:36-58``)."""
    base = (2.0 * alpha / math.pi) ** 0.75
    if l == 0:
        return float(base)
    return float(base * math.sqrt((4.0 * alpha) ** l / double_factorial(2 * l - 1)))


def contraction_norm(exponents, coeffs, l: int) -> float:
    """1/sqrt(<chi|chi>) of a contracted shell (``normalize.py:61-88``)."""
    exponents = np.asarray(exponents, dtype=np.float64)
    coeffs = np.asarray(coeffs, dtype=np.float64)
    asum = exponents[:, None] + exponents[None, :]
    pref = (math.pi / asum) ** 1.5
    ang = double_factorial(2 * l - 1) / (2.0 * asum) ** l if l > 0 else 1.0
    total = float(np.sum(coeffs[:, None] * coeffs[None, :] * pref * ang))
    if total <= 0.0:
        raise ValueError(
            f"Non-positive self-overlap ({total}) for contracted shell with l={l}."
        )
    return 1.0 / math.sqrt(total)


def normalize_shell(exponents, coeffs, l: int) -> np.ndarray:
    """d_i * N_i * M (``normalize.py:91-107``)."""
    exponents = np.asarray(exponents, dtype=np.float64)
    coeffs = np.asarray(coeffs, dtype=np.float64)
    pn = np.array([primitive_norm(float(a), l) for a in exponents])
    c = coeffs * pn
    return c * contraction_norm(exponents, c, l)


# ---------------------------------------------------------------------------
# basis library (BSE schema)
# ---------------------------------------------------------------------------


def _shell(l: int, exps, coefs) -> dict:
    return {
        "angular_momentum": [int(l)],
        "exponents": [repr(float(a)) for a in exps],
        "coefficients": [[repr(float(c)) for c in coefs]],
    }


def _geom(a0: float, ratio: float, n: int) -> List[float]:
    return [a0 * ratio**k for k in range(n)]


def _bump(n: int, centre: float, width: float) -> List[float]:
    return [math.exp(-(((k - centre) / width) ** 2)) for k in range(n)]


_STO3G = real_bases()["sto-3g"]["elements"]


def _syn_sto3g() -> dict:
    """STO-3G-shaped: H 1s(3); O 1s(3), 2s(3), 2p(3) sharing exponents."""
    o_core = _geom(131.0, 0.18, 3)
    o_val = _geom(5.2, 0.30, 3)
    return {
        "1": _STO3G["1"],
        "2": _STO3G["2"],
        "8": {
            "electron_shells": [
                _shell(0, o_core, _bump(3, 1.2, 1.1)),
                _shell(0, o_val, [-0.10, 0.40, 0.70]),
                _shell(1, o_val, [0.16, 0.60, 0.40]),
            ]
        },
    }


def _syn_631gs(h_p: bool) -> dict:
    """6-31G*-shaped (Cartesian d): H s(3) s(1) [p(1)]; O s(6) sp(3) sp(1) d(1)."""
    h_shells = [
        _shell(0, _geom(18.5, 0.16, 3), _bump(3, 1.6, 1.0)),
        _shell(0, [0.155], [1.0]),
    ]
    if h_p:
        h_shells.append(_shell(1, [1.05], [1.0]))
    o_core = _geom(5300.0, 0.205, 6)
    o_val = _geom(14.5, 0.235, 3)
    return {
        "1": {"electron_shells": h_shells},
        "8": {
            "electron_shells": [
                _shell(0, o_core, _bump(6, 3.4, 1.5)),
                _shell(0, o_val, [-0.12, -0.16, 1.08]),
                _shell(1, o_val, _bump(3, 1.4, 1.1)),
                _shell(0, [0.27], [1.0]),
                _shell(1, [0.27], [1.0]),
                _shell(2, [0.80], [1.0]),
            ]
        },
    }


_LIBRARY: Dict[str, dict] = {
    **real_bases(),
    "syn-sto-3g": {"elements": _syn_sto3g()},
    "syn-6-31g*": {"elements": _syn_631gs(False)},
    "syn-6-31g**": {"elements": _syn_631gs(True)},
}


def register_basis(name: str, bse_dict: dict) -> None:
    """Make a BSE-schema dict available under ``name``."""
    _LIBRARY[name.lower()] = bse_dict


def get_basis_dict(name: str) -> dict:
    key = name.lower()
    if key not in _LIBRARY:
        raise KeyError(f"Unknown basis {name!r}; known: {sorted(_LIBRARY)}")
    return _LIBRARY[key]


# ---------------------------------------------------------------------------
# parsing (jax_qc/basis/parse.py)
# ---------------------------------------------------------------------------


def parse_electron_shell(shell_dict: dict, center, atom_index: int) -> List[Shell]:
    """One BSE entry -> shells, one per (l, coefficient row) (``parse.py:26-89``)."""
    ams = list(shell_dict["angular_momentum"])
    exps = np.array([float(s) for s in shell_dict["exponents"]], dtype=np.float64)
    rows = shell_dict["coefficients"]
    if len(ams) == len(rows):
        pairs = list(zip(ams, rows))
    elif len(ams) == 1:
        pairs = [(ams[0], r) for r in rows]
    else:
        raise ValueError(
            "Unexpected BSE shell layout: "
            f"{len(ams)} angular momenta, {len(rows)} coefficient rows."
        )
    out = []
    for l, row in pairs:
        c = np.array([float(s) for s in row], dtype=np.float64)
        mask = c != 0.0
        a = exps[mask] if not mask.all() else exps
        c = c[mask] if not mask.all() else c
        out.append(
            Shell(
                angular_momentum=int(l),
                exponents=a.copy(),
                coefficients=normalize_shell(a, c, int(l)),
                center=np.asarray(center, dtype=np.float64).copy(),
                atom_index=int(atom_index),
            )
        )
    return out


def bse_dict_to_shells(bse_data: dict, mol) -> List[Shell]:
    """All shells of ``mol`` in atom order, sorted per atom by (l, -max exp)
    (``parse.py:92-127``)."""
    shells: List[Shell] = []
    elements = bse_data.get("elements", {})
    Z = np.asarray(mol.atomic_numbers).tolist()
    coords = np.asarray(mol.coords, dtype=np.float64)
    for ia, z in enumerate(Z):
        key = str(int(z))
        if key not in elements:
            raise KeyError(f"Basis set does not define element Z={z} (atom index {ia}).")
        atom_shells: List[Shell] = []
        for sd in elements[key].get("electron_shells", []):
            atom_shells.extend(parse_electron_shell(sd, coords[ia], ia))
        atom_shells.sort(key=lambda s: (int(s.angular_momentum), -float(np.max(s.exponents))))
        shells.extend(atom_shells)
    return shells


def build_shell_indices(shells, spherical: bool = True):
    """(shell_to_basis, basis_to_atom, n_basis) (``parse.py:130-152``)."""
    s2b, b2a, off = [], [], 0
    for sh in shells:
        l = int(sh.angular_momentum)
        n = (2 * l + 1) if spherical else n_cartesian(l)
        s2b.append(tuple(range(off, off + n)))
        b2a.extend([int(sh.atom_index)] * n)
        off += n
    return tuple(s2b), np.asarray(b2a, dtype=np.int32), off


def build_basis_set(mol, basis, spherical: bool = False) -> BasisSet:
    """Build a BasisSet for ``mol`` (``jax_qc/basis/build.py:24-62``).

    ``basis`` is a registered name or a BSE-schema dict.  The default here is
    Cartesian (``spherical=False``), the layout the two-electron kernels work
    in; spherical sets are handled by an N^2 transform of D/J/K.
    """
    data = basis if isinstance(basis, dict) else get_basis_dict(basis)
    name = basis if isinstance(basis, str) else str(data.get("name", "custom"))
    shells = bse_dict_to_shells(data, mol)
    s2b, b2a, n = build_shell_indices(shells, spherical=spherical)
    return BasisSet(
        shells=tuple(shells),
        n_basis=n,
        shell_to_basis=s2b,
        basis_to_atom=b2a,
        name=name,
        spherical=spherical,
    )


# ---------------------------------------------------------------------------
# test systems: water monomer and seeded water clusters
# ---------------------------------------------------------------------------

WATER_OH_ANGSTROM = 0.9572
WATER_HOH_DEGREES = 104.52


def water_monomer_bohr() -> np.ndarray:
    """O at the origin, H atoms in the xz plane; O-H 0.9572 A, H-O-H 104.52 deg."""
    r = WATER_OH_ANGSTROM * ANGSTROM_TO_BOHR
    half = math.radians(WATER_HOH_DEGREES) / 2.0
    return np.array(
        [
            [0.0, 0.0, 0.0],
            [r * math.sin(half), 0.0, r * math.cos(half)],
            [-r * math.sin(half), 0.0, r * math.cos(half)],
        ]
    )


def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))[None, :]
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def lattice_shape(n_waters: int):
    """Cubic-lattice extents used for the water clusters: 2x2x2 for 8, 2x2x4
    for 16, otherwise the smallest near-cubic box holding ``n_waters``."""
    if n_waters == 8:
        return (2, 2, 2)
    if n_waters == 16:
        return (2, 2, 4)
    a = max(1, int(math.ceil(n_waters ** (1.0 / 3.0) - 1e-9)))
    for shape in ((a, a - 1, a - 1), (a, a, a - 1), (a, a, a)):
        if min(shape) > 0 and shape[0] * shape[1] * shape[2] >= n_waters:
            return shape
    return (a, a, a)


def water_cluster(
    n_waters: int,
    seed: int = 0,
    spacing_angstrom: float = 2.9,
    noise_angstrom: float = 0.0,
    charge: int = 0,
    spin: int = 0,
) -> Molecule:
    """(H2O)_n on a cubic lattice (``spacing_angstrom``) with seeded random
    rotations of the monomer about O, plus optional Gaussian coordinate noise."""
    if n_waters < 1:
        raise ValueError("n_waters must be >= 1")
    rng = np.random.default_rng(seed)
    mono = water_monomer_bohr()
    nx, ny, nz = lattice_shape(n_waters)
    a = spacing_angstrom * ANGSTROM_TO_BOHR
    coords, elements, Z = [], [], []
    k = 0
    for iz in range(nz):
        for iy in range(ny):
            for ix in range(nx):
                if k == n_waters:
                    break
                rot = _random_rotation(rng) if n_waters > 1 else np.eye(3)
                origin = np.array([ix * a, iy * a, iz * a])
                coords.append(mono @ rot.T + origin)
                elements += ["O", "H", "H"]
                Z += [8, 1, 1]
                k += 1
    xyz = np.concatenate(coords, axis=0)
    if noise_angstrom > 0.0:
        xyz = xyz + rng.standard_normal(xyz.shape) * noise_angstrom * ANGSTROM_TO_BOHR
    return make_molecule(tuple(elements), xyz, np.array(Z, dtype=np.int32), charge=charge, spin=spin)
