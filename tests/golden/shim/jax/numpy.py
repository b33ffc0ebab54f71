"""``jax.numpy`` for the test shim: plain NumPy."""
from numpy import *  # noqa: F401,F403
from numpy import linalg, ndarray, pi  # noqa: F401
