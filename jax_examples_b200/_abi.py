"""ctypes binding of libjqc.so (the C ABI declared in include/jqc.h).

The library must have been built in-tree (``__graft_entry__.build()`` or
``python -m jax_examples_b200._build``).  There is no fallback: a missing
library or a failed call raises.  Status codes map onto the exceptions the
reference raises for the same conditions (ValueError for bad input,
NotImplementedError for unsupported angular momentum).
"""

from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libjqc.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "jqc.h")

JQC_OK = 0
JQC_ERR_INVALID = 1
JQC_ERR_CUDA = 2
JQC_ERR_TOO_LARGE = 3
JQC_ERR_NOT_READY = 4
JQC_ERR_UNSUPPORTED = 5
JQC_ERR_TIMEOUT = 6

PREC = {"fp64": 0, "mixed": 1, "fp32": 2}


class JQCError(RuntimeError):
    """A libjqc call failed (CUDA error or call-order violation)."""


class JQCTooLarge(ValueError):
    """The requested dense output exceeds its size cap."""


class JQCTimeout(TimeoutError):
    """A bounded device-side wait gave up."""


_c_int = ctypes.c_int
_c_ll = ctypes.c_longlong
_c_dbl = ctypes.c_double
_vp = ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)
_llp = ctypes.POINTER(ctypes.c_longlong)

# name -> (restype, argtypes)
SIGNATURES = {
    "jqc_last_error": (ctypes.c_char_p, []),
    "jqc_version": (_c_int, []),
    "jqc_ctx_create": (_c_int, [_c_int, ctypes.POINTER(_vp)]),
    "jqc_ctx_destroy": (_c_int, [_vp]),
    "jqc_basis_upload": (_c_int, [_vp, _c_int, _ip, _ip, _ip, _dp, _dp, _dp, _ip, _c_int, _dp, _dp, _c_int]),
    "jqc_pairs_build": (_c_int, [_vp, _c_dbl, _c_dbl, _vp]),
    "jqc_stats": (_c_int, [_vp, _c_int, _c_dbl, _llp]),
    "jqc_schwarz": (_c_int, [_vp, _vp, _vp]),
    "jqc_boys": (_c_int, [_vp, _c_ll, _c_int, _vp, _c_int, _vp]),
    "jqc_eri_prim_quartets": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_ll, _vp, _vp, _vp, _vp]),
    "jqc_eri_tensor": (_c_int, [_vp, _vp, _c_ll, _vp]),
    "jqc_one_electron": (_c_int, [_vp, _vp, _vp, _vp, _vp]),
    "jqc_jk": (_c_int, [_vp, _c_int, _vp, _vp, _vp, _c_int, _c_dbl, _c_dbl, _vp]),
    "jqc_grad2e": (_c_int, [_vp, _c_int, _vp, _c_dbl, _c_dbl, _vp, _vp]),
    "jqc_grad1e": (_c_int, [_vp, _vp, _vp, _vp, _vp]),
    "jqc_jk_noalloc": (_c_int, [_vp, _c_int, _vp, _vp, _vp, _c_int, _c_dbl, _c_dbl, _vp]),
    "jqc_jk_timed": (_c_int, [_vp, _c_int, _vp, _vp, _vp, _c_int, _c_dbl, _c_dbl, _vp, _dp]),
    "jqc_class_stats": (_c_int, [_vp, _c_int, _c_dbl, _llp]),
    "jqc_fp_peak": (_c_int, [_c_int, _c_int, _c_int, _dp, _vp]),
    "jqc_batch_partition": (_c_int, [_vp, _c_int, _ip]),
    "jqc_set_geometry": (_c_int, [_vp, _dp]),
    "jqc_set_molecule_mask": (_c_int, [_vp, _ip]),
    "jqc_set_molecule_activity": (_c_int, [_vp, _vp]),
    "jqc_grad2e_ex": (_c_int, [_vp, _c_int, _vp, _c_dbl, _c_dbl, _c_dbl, _vp, _vp, _dp]),
    "jqc_set_grad_engine": (_c_int, [_vp, _c_int, _c_int]),
    "jqc_get_grad_engine": (_c_int, [_vp, _ip]),
    "jqc_graph_begin": (_c_int, [_vp, _vp]),
    "jqc_graph_end": (_c_int, [_vp, _vp, ctypes.POINTER(_c_int)]),
    "jqc_graph_launch": (_c_int, [_vp, _c_int, _vp]),
    "jqc_graph_destroy": (_c_int, [_vp, _c_int]),
    "jqc_get_tuning": (_c_int, [_vp, _ip]),
    "jqc_set_tuning": (_c_int, [_vp, _ip]),
    "jqc_autotune": (_c_int, [_vp, _c_int, _vp, _vp, _vp, _c_int, _c_dbl, _c_dbl, ctypes.c_char_p,
                              ctypes.POINTER(_c_int), _vp]),
}

_LIB = None


def header_symbols(path: str = HEADER):
    """Function names declared in include/jqc.h."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jqc_[a-z0-9_]+)\s*\(", text)))


def load() -> ctypes.CDLL:
    """Load libjqc.so and attach signatures; raises if it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m jax_examples_b200._build` "
            "(there is no CPU fallback for the two-electron path)"
        )
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def check(rc: int, what: str) -> None:
    if rc == JQC_OK:
        return
    msg = load().jqc_last_error().decode(errors="replace")
    text = f"{what}: {msg}"
    if rc == JQC_ERR_INVALID:
        raise ValueError(text)
    if rc == JQC_ERR_UNSUPPORTED:
        raise NotImplementedError(text)
    if rc == JQC_ERR_TOO_LARGE:
        raise JQCTooLarge(text)
    if rc == JQC_ERR_TIMEOUT:
        raise JQCTimeout(text)
    raise JQCError(f"{text} (status {rc})")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)
