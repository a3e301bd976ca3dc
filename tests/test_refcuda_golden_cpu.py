"""CPU tests against committed outputs of the reference's own CUDA kernel
(tests/golden/refcuda_vectors.npz, made on a B200 by
tests/golden/make_refcuda_golden.py from cuda/ncs.cu compiled unmodified).

They replay, without a GPU, the reference's own GPU-vs-C checks with the
oracle standing in for the C side: the seed(1) tiles of
cuda/pyCUDANCS/test/test_solver.py (max |u_gpu - u_c| / max |u_c| < 1e-2
per tile, :116-118) and the 30 x 30 image of cuda/pyCUDANCS/test/test_im.py
(atol 0.02, :42).  They also hold the oracle's FP64 Newton referee against
the kernel's converged tiles.
"""
import os

import numpy
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "refcuda_vectors.npz")


@pytest.fixture(scope="module")
def gold():
    if not os.path.exists(GOLD):
        pytest.skip("reference CUDA kernel vectors not generated")
    return dict(numpy.load(GOLD))


def test_c_solver_matches_the_cuda_kernel_on_tiles(gold, oracle_libs):
    # test_solver.py:99-118: each tile solved by the C solver (the compiled
    # reference ncs.c when present, else our C port) against the kernel's
    d, g = gold["tiles_data"].astype(numpy.float64), gold["tiles_gamma"].astype(numpy.float64)
    ms = gold["tiles_mask_shifted"].astype(numpy.float64)
    alpha = float(gold["tiles_alpha"])
    u_gpu = gold["tiles_u"]
    assert (gold["tiles_status"] == 0).all()
    for i in range(d.shape[0]):
        u_c, _, _ = oracle_libs.solve_tile(d[i], g[i], ms, alpha)
        assert numpy.abs(u_gpu[i] - u_c).max() / numpy.abs(u_c).max() < 1e-2, i


def test_fp64_referee_agrees_with_the_cuda_kernel(gold):
    # the kernel stops at ||g|| <= 1e-4 max(||u||, 1) in FP32 (ncs.cu:55):
    # its converged tiles lie within 1e-6 relative cost of the FP64 optimum
    from oracle import numpy_ref as nr
    d, g = gold["tiles_data"].astype(numpy.float64), gold["tiles_gamma"].astype(numpy.float64)
    ms = gold["tiles_mask_shifted"].astype(numpy.float64)
    alpha = float(gold["tiles_alpha"])
    ustar, fstar, _ = nr.newton_solve(d, g, ms, alpha)
    f_gpu = nr.cost(gold["tiles_u"].astype(numpy.float64), d, g, ms, alpha)
    assert nr.rel_cost_gap(f_gpu, fstar).max() <= 1e-6
    rel = numpy.abs(gold["tiles_u"] - ustar) / numpy.maximum(numpy.abs(ustar), 1.0)
    assert rel.max() <= 1e-2


def test_c_image_path_matches_the_cuda_kernel(gold, oracle_libs):
    # test_im.py:31-42 at (ix, iy) = (0, 0): cReduceNoise against the kernel's
    # segmented, solved and stitched image
    image = gold["image"].astype(numpy.float64)
    gam = gold["image_gamma"].astype(numpy.float64)
    ms = gold["image_mask_shifted"].astype(numpy.float64)
    ncs1 = oracle_libs.cReduceNoise(image, gam, ms, float(gold["image_alpha"]))
    assert numpy.allclose(ncs1, gold["image_out"], atol=0.02)
