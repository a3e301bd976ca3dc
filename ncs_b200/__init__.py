"""ncs_b200 -- B200-native NCS (sCMOS noise correction) per-tile L-BFGS solver.

The compute path is libncs_b200.so (hand-written sm_100a CUDA behind the C
ABI of include/ncs_b200.h), loaded with ctypes.  Importing this package loads
it; there is no CPU fallback.
"""
from . import _lib
from .ncs import (NCSCUDA, NCSCUDAException, Solver, cReduceNoise, checkOTFMask,
                  reduce_noise_normalized, reduceNoise)

_lib.load()

__all__ = ["Solver", "NCSCUDA", "NCSCUDAException", "reduceNoise", "cReduceNoise",
           "reduce_noise_normalized",
           "checkOTFMask"]
