"""CPU oracle for the NCS per-tile solve -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm may import this package, and only as the checker or as the
timed CPU reference.  The shipped CUDA path (``ncs_b200``) never imports it
and has no CPU fallback.

Contents:
  * ``lib/libncs_port.so``  -- our FP64 C restatement of ``clib/pyCNCS/ncs.c``.
  * ``_ref/libncs.so``      -- the reference's own ``ncs.c`` compiled unmodified
    against our FFTW-API shim and libLBFGS-API solver (``Makefile``).
  * ``pycncs``              -- ctypes bindings mirroring ``clib/pyCNCS/ncs_c.py``.
  * ``numpy_ref``           -- FP64 numpy restatements (cost, gradient, the
    quadratic form Q, segmentation/stitching, exact Newton optimum).
"""
