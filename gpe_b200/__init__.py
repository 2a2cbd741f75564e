"""gpe_b200 -- a B200 (sm_100a) finite-difference time stepper for the
Gross-Pitaevskii equation, drop-in for the hot path of liangjj/gpe.

The compute path is ``libgpe_gpu.so`` (hand-written CUDA, C-ABI in
include/gpe_gpu.h); this package is its host-side mirror of the reference's
solver module.  Importing the package does not load the library; the first
call that needs it does, and raises if it is missing.
"""
from ._lib import GpeError, LIB_PATH, lib  # noqa: F401
from .solver import GpeParams, GpeSolver, run_loop  # noqa: F401
from .batch import BatchOpts, GpeBatch  # noqa: F401

__all__ = ["GpeError", "GpeParams", "GpeSolver", "run_loop", "lib", "LIB_PATH"]
