"""The reference's CUDA kernel on the GPU -- TEST INFRASTRUCTURE ONLY.

``cuda/ncs.cu`` (``ncsReduceNoise``) compiled unmodified for sm_100a by
``oracle/Makefile`` into ``_ref/libncs_ref_cuda.so`` (with our float4
operator header standing in for the CUDA samples' absent helper_math.h), and
driven the way ``cuda/pyCUDANCS/ncs.py:38-171`` drives it, with the host loops
done as torch indexing on the device:
  * ``segment`` -- edge-replicated tiles at the origins of ncs.py:81-98,
  * ``reduce_noise_tiles`` -- one 16-thread block per tile (ncs.py:116-125),
  * ``stitch`` -- interiors back in tile order, later tiles overwriting
    (ncs.py:161-169).
Used by the GPU tests as a second, GPU-side check of our kernels and by the
benchmark's reference arm to time the reference's own GPU path.
"""
import ctypes
import os

import numpy
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libncs_ref_cuda.so")
R = 16

_lib = None


def available():
    return os.path.exists(LIB)


def load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        lib.ref_cuda_reduce_noise_tiles.argtypes = [vp, vp, vp, vp, vp, vp, ctypes.c_float,
                                                    ctypes.c_longlong, vp]
        lib.ref_cuda_reduce_noise_tiles.restype = ctypes.c_int
        _lib = lib
    return _lib


def origins(n):
    """Tile origins along an axis of n pixels in padded coordinates
    (ncs.py:82-86: i = 0, 14, 28, ... over n + 2, the last one moved back so
    that it ends at the padded edge)."""
    out = []
    for i in range(0, n + 2, R - 2):
        out.append(n + 2 - R if i + R > n + 2 else i)
    return out


def segment(images, gamma):
    """[T, H, W] CUDA stack and gamma [H, W] -> data, gamma tiles
    [T * nx * ny, 16, 16] in (frame, row origin, column origin) order."""
    T, H, W = images.shape
    dev = images.device
    ox = torch.tensor(origins(H), device=dev)
    oy = torch.tensor(origins(W), device=dev)
    ar = torch.arange(R, device=dev)
    rows = (ox[:, None] + ar)[:, None, :, None]   # [nx, 1, 16, 1]
    cols = (oy[:, None] + ar)[None, :, None, :]   # [1, ny, 1, 16]
    pad = torch.nn.functional.pad(images[:, None], (1, 1, 1, 1), mode="replicate")[:, 0]
    data = pad[:, rows, cols].reshape(-1, R, R).contiguous()
    gpad = torch.nn.functional.pad(gamma[None, None], (1, 1, 1, 1), mode="replicate")[0, 0]
    gt = gpad[rows, cols].reshape(1, -1, R, R).expand(T, -1, R, R).reshape(-1, R, R)
    return data, gt.contiguous()


def stitch(tiles, shape):
    """Tile interiors back into a [T, H, W] stack: each pixel from the last
    tile (in tile order) whose interior covers it."""
    T, H, W = shape
    dev = tiles.device

    def owners(n):
        org = origins(n)
        own = numpy.zeros(n, dtype=numpy.int64)
        off = numpy.zeros(n, dtype=numpy.int64)
        for k, o in enumerate(org):       # later tiles overwrite
            own[o:o + R - 2] = k
            off[o:o + R - 2] = numpy.arange(R - 2) + 1
        return (torch.from_numpy(own).to(dev), torch.from_numpy(off).to(dev), len(org))
    orow, frow, nx = owners(H)
    ocol, fcol, ny = owners(W)
    t = tiles.reshape(T, nx, ny, R, R)
    return t[:, orow[:, None], ocol[None, :], frow[:, None], fcol[None, :]]


def reduce_noise_tiles(data, gamma, mask_shifted, alpha, stream=None):
    """Run ncsReduceNoise on [N, 16, 16] FP32 CUDA tiles.  mask_shifted: the
    16 x 16 mask with DC at [0, 0] (ncs.py:197).  Returns (out, iterations,
    status), the kernel's own outputs."""
    lib = load()
    n = data.shape[0]
    dev = data.device
    mask = torch.as_tensor(numpy.asarray(mask_shifted, dtype=numpy.float32)).to(dev).contiguous()
    out = torch.empty_like(data)
    iters = torch.zeros(n, dtype=torch.int32, device=dev)
    status = torch.zeros(n, dtype=torch.int32, device=dev)
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    with torch.cuda.device(dev):
        rc = lib.ref_cuda_reduce_noise_tiles(data.data_ptr(), gamma.data_ptr(), mask.data_ptr(),
                                             out.data_ptr(), iters.data_ptr(), status.data_ptr(),
                                             float(alpha), n, ctypes.c_void_p(s.cuda_stream))
    if rc != 0:
        raise RuntimeError("reference CUDA kernel launch failed: cuda error %d" % rc)
    return out, iters, status
