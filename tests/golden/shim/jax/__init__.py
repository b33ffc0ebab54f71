"""Test-only stand-in for ``jax`` so the reference ``jax_qc`` package imports in
a container that has no JAX.  ``jax.numpy`` is NumPy, ``jax.lax.erf`` is
``scipy.special.erf``; ``jit`` is the identity and the config/barrier calls are
no-ops.  Used only by ``tests/golden/gen_golden.py`` to run the reference's own
FP64 code and record golden vectors.  Never imported by the product."""

from . import lax  # noqa: F401
from . import numpy  # noqa: F401


class _Config:
    def update(self, *args, **kwargs):
        return None


config = _Config()


def jit(fn, *args, **kwargs):
    return fn


def effects_barrier():
    return None


def grad(*args, **kwargs):  # the reference never calls it on the traced path
    raise NotImplementedError("jax.grad is not available in the test shim")
