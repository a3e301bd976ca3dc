"""ncs_b200 -- B200-native NCS (sCMOS noise correction) per-tile L-BFGS solver.

The compute path is libncs_b200.so (hand-written sm_100a CUDA behind the C
ABI of include/ncs_b200.h), loaded with ctypes on the first call that needs
it.  Importing the package checks that the library is built and raises if
not; there is no CPU fallback.
"""
from . import _lib
from .ncs import (NCSCUDA, NCSCUDAException, Solver, cReduceNoise, checkOTFMask,
                  reduce_noise_normalized, reduceNoise)

_lib.require()

__all__ = ["Solver", "NCSCUDA", "NCSCUDAException", "reduceNoise", "cReduceNoise",
           "reduce_noise_normalized",
           "checkOTFMask"]
