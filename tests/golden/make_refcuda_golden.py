"""Generate tests/golden/refcuda_vectors.npz: outputs of the reference's own
CUDA kernel (cuda/ncs.cu ncsReduceNoise, compiled unmodified for sm_100a by
oracle/Makefile into oracle/_ref/libncs_ref_cuda.so), so that CPU tests can
hold the oracle against the reference GPU path without a GPU.

Needs a B200 and the built kernel.  Usage:

    python tests/golden/make_refcuda_golden.py OUT.npz

Cases (inputs stored beside the outputs):
  * tiles: the 64 seed(1) tiles of cuda/pyCUDANCS/test/test_solver.py:79-84
    (data U(10, 20), gamma U(2, 4)), alpha 0.1, the Gaussian high-pass mask
    of opencl/pyOpenCLNCS/py_ref.py:129-137 (fftshifted).
  * image: the 30 x 30 seed(1) image of cuda/pyCUDANCS/test/test_im.py:22-29
    (image U(0.01, 10), gamma U(2, 4)), alpha 0.02, a random symmetric mask
    (clib/pyCNCS/test/py_ref.py:77-85 recipe, numpy default_rng(1)), cut,
    solved and stitched as cuda/pyCUDANCS/ncs.py does.
"""
import os
import sys

import numpy
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from conftest import create_otf_mask_shifted, random_otf_mask  # noqa: E402
from oracle import refgpu  # noqa: E402


def main(out_path):
    assert torch.cuda.is_available() and refgpu.available()
    # tiles (test_solver.py)
    n, alpha_t = 64, 0.1
    numpy.random.seed(1)
    tiles = numpy.random.uniform(10.0, 20.0, size=(n, 16, 16)).astype(numpy.float32)
    tgam = numpy.random.uniform(2.0, 4.0, size=(n, 16, 16)).astype(numpy.float32)
    tmask = create_otf_mask_shifted()
    u, it, st = refgpu.reduce_noise_tiles(torch.from_numpy(tiles).cuda(),
                                          torch.from_numpy(tgam).cuda(), tmask, alpha_t)
    # image (test_im.py)
    im_size, alpha_i = 30, 0.02
    numpy.random.seed(1)
    igam = numpy.random.uniform(2.0, 4.0, size=(im_size, im_size)).astype(numpy.float32)
    image = numpy.random.uniform(0.01, 10.0, size=(im_size, im_size)).astype(numpy.float32)
    imask = numpy.fft.fftshift(random_otf_mask(16, numpy.random.default_rng(1))).astype(
        numpy.float32)
    x = torch.from_numpy(image).cuda()[None]
    dt, gt = refgpu.segment(x, torch.from_numpy(igam).cuda())
    ui, iti, sti = refgpu.reduce_noise_tiles(dt, gt, imask, alpha_i)
    out = refgpu.stitch(ui, x.shape)[0]
    torch.cuda.synchronize()
    numpy.savez_compressed(
        out_path,
        tiles_data=tiles, tiles_gamma=tgam, tiles_mask_shifted=tmask, tiles_alpha=alpha_t,
        tiles_u=u.cpu().numpy(), tiles_iters=it.cpu().numpy(), tiles_status=st.cpu().numpy(),
        image=image, image_gamma=igam, image_mask_shifted=imask, image_alpha=alpha_i,
        image_out=out.cpu().numpy(), image_status=sti.cpu().numpy(),
        kernel="cuda/ncs.cu ncsReduceNoise, unmodified, nvcc -gencode "
               "arch=compute_100a,code=sm_100a -O3, B200")
    print("wrote", out_path)


if __name__ == "__main__":
    main(sys.argv[1])
