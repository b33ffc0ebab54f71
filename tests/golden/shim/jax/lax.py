"""``jax.lax`` for the test shim: only ``erf`` is used by the reference."""
from scipy.special import erf  # noqa: F401
