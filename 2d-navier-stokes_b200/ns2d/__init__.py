"""ns2d -- B200 pseudospectral step of the 2-D vorticity Navier-Stokes solver.

Python side of libns2d.so (include/ns2d.h).  `abi` holds the C types; `Solver`
mirrors the reference's per-step C functions; `initial` builds seeded test
inputs.
"""
from . import abi
from ._lib import NS2DError, load, LIB_PATH
from .solver import Solver
from .ensemble import Ensemble

__all__ = ["abi", "Solver", "Ensemble", "NS2DError", "load", "LIB_PATH"]
