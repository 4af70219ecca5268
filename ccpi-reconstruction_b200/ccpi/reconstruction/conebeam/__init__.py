"""Cone-beam reconstruction (drop-in for the reference's
``ccpi.reconstruction.conebeam`` extension module)."""
from . import alg  # noqa: F401
