"""Parallel-beam reconstruction (drop-in for the reference's
``ccpi.reconstruction.parallelbeam`` extension module)."""
from . import alg  # noqa: F401
from . import filters  # noqa: F401
