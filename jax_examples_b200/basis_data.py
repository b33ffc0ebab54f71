"""Published Gaussian basis-set parameters as BSE-schema dicts.

The Basis Set Exchange (``basis_set_exchange``, which the reference fetches
through ``jax_qc/basis/bse_fetch.py:15-60``) is not installed, so the bases the
two-electron workloads name are carried here as constant tables, in the schema
``get_basis(..., uncontract_spdf=True)`` returns (one entry per shell, an
``sp`` shell as two coefficient rows over shared exponents, which
``bse_dict_to_shells`` splits into an s and a p shell):

* STO-3G for H, C, N, O, F (Hehre, Stewart and Pople, J. Chem. Phys. 51,
  2657 (1969)): the three-Gaussian fits of Slater 1s and 2sp functions with
  exponent 1 (shared contraction coefficients), scaled by each element's
  Slater exponent squared.
* 6-31G for H and O (Hehre, Ditchfield and Pople, J. Chem. Phys. 56, 2257
  (1972)); 6-31G* adds one d shell (exponent 0.8) on O (Hariharan and Pople,
  Theor. Chim. Acta 28, 213 (1973)); 6-31G** adds one p shell (exponent 1.1)
  on H.

Coefficients are those of normalized primitives, as BSE distributes them; the
basis layer normalizes the contractions the way the reference does
(``jax_qc/basis/normalize.py:91-107``).  The transcription is pinned by the
PySCF RHF energies the reference carries for water, HF, CH4 and NH3
(``examples/08_rhf_tier2.py:33-41``) and by energies of the reference's own
code on the same tables.
"""

from __future__ import annotations

from typing import Dict, List


def _sh(ams: List[int], exps: List[float], rows: List[List[float]]) -> dict:
    return {
        "function_type": "gto",
        "angular_momentum": list(ams),
        "exponents": [repr(float(a)) for a in exps],
        "coefficients": [[repr(float(c)) for c in r] for r in rows],
    }


# --------------------------------------------------------------------- STO-3G
# Contraction coefficients of the 1s and 2sp three-Gaussian fits (shared by
# every element) and the element exponents, to the eight significant digits
# of the published tables.
_STO3G_1S = [0.15432897, 0.53532814, 0.44463454]
_STO3G_2S = [-0.09996723, 0.39951283, 0.70011547]
_STO3G_2P = [0.15591627, 0.60768372, 0.39195739]

_STO3G_EXPS = {
    1: ([3.42525091, 0.62391373, 0.16885540], None),
    6: ([71.6168370, 13.0450960, 3.5305122], [2.9412494, 0.6834831, 0.2222899]),
    7: ([99.1061690, 18.0523120, 4.8856602], [3.7804559, 0.8784966, 0.2857144]),
    8: ([130.7093200, 23.8088610, 6.4436083], [5.0331513, 1.1695961, 0.3803890]),
    9: ([166.6791300, 30.3608120, 8.2168207], [6.4648032, 1.5022812, 0.4885885]),
}


def _sto3g() -> dict:
    elements: Dict[str, dict] = {}
    for z, (e1s, e2sp) in _STO3G_EXPS.items():
        shells = [_sh([0], e1s, [_STO3G_1S])]
        if e2sp is not None:
            shells.append(_sh([0, 1], e2sp, [_STO3G_2S, _STO3G_2P]))
        elements[str(z)] = {"electron_shells": shells}
    # He as the reference carries it (fp/qchem_fp.py:64-76).
    elements["2"] = {"electron_shells": [_sh([0], [6.36242139, 1.15892300, 0.31364979], [_STO3G_1S])]}
    return {"name": "sto-3g", "elements": elements}


# ---------------------------------------------------------------------- 6-31G
_H_631G = [
    _sh([0], [18.7311370, 2.8253937, 0.6401217], [[0.03349460, 0.23472695, 0.81375733]]),
    _sh([0], [0.1612778], [[1.0]]),
]
_O_631G = [
    _sh([0], [5484.6717000, 825.2349500, 188.0469600, 52.9645000, 16.8975700, 5.7996353],
        [[0.0018311, 0.0139501, 0.0684451, 0.2327143, 0.4701930, 0.3585209]]),
    _sh([0, 1], [15.5396160, 3.5999336, 1.0137618],
        [[-0.1107775, -0.1480263, 1.1307670], [0.0708743, 0.3397528, 0.7271586]]),
    _sh([0, 1], [0.2700058], [[1.0], [1.0]]),
]
_O_D = _sh([2], [0.8], [[1.0]])
_H_P = _sh([1], [1.1], [[1.0]])


def _631g(o_d: bool, h_p: bool) -> dict:
    h = list(_H_631G) + ([_H_P] if h_p else [])
    o = list(_O_631G) + ([_O_D] if o_d else [])
    return {"elements": {"1": {"electron_shells": h}, "8": {"electron_shells": o}}}


def real_bases() -> Dict[str, dict]:
    """Name -> BSE-schema dict for every published basis carried here."""
    out = {
        "sto-3g": _sto3g(),
        "6-31g": _631g(False, False),
        "6-31g*": _631g(True, False),
        "6-31g**": _631g(True, True),
    }
    for name, d in out.items():
        d["name"] = name
    return out
