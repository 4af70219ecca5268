"""Parallel-beam reconstruction (drop-in for the reference's
``ccpi.reconstruction.parallelbeam`` extension module)."""
from . import alg  # noqa: F401
