"""Oracle for the NCS per-tile solve -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline,
accuracy and reference legs may import this package, and only as the checker
or as the timed reference implementation.  The shipped CUDA path
(``ncs_b200``) never imports it and has no CPU fallback.

Contents:
  * ``lib/libncs_port.so``  -- our FP64 C restatement of ``clib/pyCNCS/ncs.c``.
  * ``_ref/libncs.so``      -- the reference's own ``ncs.c`` compiled unmodified
    against our FFTW-API shim and libLBFGS-API solver (``Makefile``).
  * ``pycncs``              -- ctypes bindings mirroring ``clib/pyCNCS/ncs_c.py``.
  * ``_ref/libncs_ref_cuda.so`` -- the reference's own CUDA kernel
    ``cuda/ncs.cu`` compiled unmodified for sm_100a (``ref_cuda/``: our float4
    operator header and a C launch entry); ``refgpu`` drives it as
    ``cuda/pyCUDANCS/ncs.py`` does.
  * ``numpy_ref``           -- FP64 numpy restatements (cost, gradient, the
    quadratic form Q, segmentation/stitching, exact Newton optimum).
  * ``gpu_mirror``, ``warmstart_ref``, ``normalized_ref`` -- restatements of
    the plain GPU algorithm, the warm-start network and the normalised
    single-pixel variant.
"""
