"""GPU tests against the reference's own CUDA kernel.

``cuda/ncs.cu`` (``ncsReduceNoise``: one 16-thread block per tile, L-BFGS
with M = 8 pairs, Armijo backtracking, stop at ||g|| <= 1e-4 max(||u||, 1),
200 iterations at most) is compiled unmodified for sm_100a by
oracle/Makefile and driven as cuda/pyCUDANCS/ncs.py drives it
(oracle/refgpu.py).  The reference's own GPU tests compare that kernel with
its C solver: max |u - u_ref| / max |u_ref| < 1e-2 per tile
(cuda/pyCUDANCS/test/test_solver.py:116-118) and atol 0.02 on stitched crops
of a 30 x 30 image (cuda/pyCUDANCS/test/test_im.py:16-44).  Here our
kernels stand where the C solver stood, with the same criteria, and both
are also held against the FP64 optimum.
"""
import numpy
import pytest
import torch

from conftest import create_otf_mask_shifted, random_otf_mask

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref(cuda_ok):
    from oracle import refgpu
    if not refgpu.available():
        pytest.skip("reference CUDA kernel not built (make -C oracle ref)")
    return refgpu


@pytest.fixture(scope="module")
def ncs(cuda_ok):
    import ncs_b200
    return ncs_b200


@pytest.mark.parametrize("mode", ["spectral", "plain", "plain_wg"])
def test_tiles_match_the_reference_kernel(ref, ncs, mode):
    from oracle import numpy_ref as nr
    # test_solver.py:79-84: seed(1), data U(10, 20), gamma U(2, 4), alpha 0.1
    n, alpha = 64, 0.1
    numpy.random.seed(1)
    data = numpy.random.uniform(10.0, 20.0, size=(n, 16, 16)).astype(numpy.float32)
    gamma = numpy.random.uniform(2.0, 4.0, size=(n, 16, 16)).astype(numpy.float32)
    ms = create_otf_mask_shifted()
    d, g = torch.from_numpy(data).cuda(), torch.from_numpy(gamma).cuda()
    u_ref, it_ref, st_ref = ref.reduce_noise_tiles(d, g, ms, alpha)
    s = ncs.Solver(alpha=alpha, mode=mode, max_iters=200)
    s.set_otf_mask_shifted(ms)
    u, it, st, _ = s.solve_tiles(d, g)
    assert (st_ref == 0).all() and (st == 0).all()
    u_ref, u = u_ref.cpu().numpy(), u.cpu().numpy()
    for i in range(n):
        assert numpy.abs(u[i] - u_ref[i]).max() / numpy.abs(u_ref[i]).max() < 1e-2
    # both against the FP64 optimum: ours at least as close as the reference
    m64 = ms.astype(numpy.float64)
    _, fstar, _ = nr.newton_solve(data, gamma, m64, alpha)
    gap = nr.rel_cost_gap(nr.cost(u.astype(numpy.float64), data.astype(numpy.float64),
                                  gamma.astype(numpy.float64), m64, alpha), fstar)
    gap_ref = nr.rel_cost_gap(nr.cost(u_ref.astype(numpy.float64), data.astype(numpy.float64),
                                      gamma.astype(numpy.float64), m64, alpha), fstar)
    assert gap.max() <= max(gap_ref.max(), 1e-6)


def test_crops_match_the_reference_kernel(ref, ncs):
    # test_im.py:16-44: 144 crops image[ix:30, iy:30], alpha 0.02, a random
    # mask, atol 0.02 -- odd sizes, shifted last tiles, repeated origins
    im_size, alpha = 30, 0.02
    numpy.random.seed(1)
    gamma = numpy.random.uniform(2.0, 4.0, size=(im_size, im_size)).astype(numpy.float32)
    image = numpy.random.uniform(0.01, 10.0, size=(im_size, im_size)).astype(numpy.float32)
    mask = random_otf_mask(16, numpy.random.default_rng(1))
    ms = numpy.fft.fftshift(mask).astype(numpy.float32)
    s = ncs.Solver(alpha=alpha, max_iters=200)
    s.set_otf_mask_shifted(ms)
    worst = 0.0
    for ix in range(12):
        for iy in range(12):
            im = torch.from_numpy(numpy.ascontiguousarray(image[ix:, iy:])).cuda()[None]
            gm = torch.from_numpy(numpy.ascontiguousarray(gamma[ix:, iy:])).cuda()
            dt, gt = ref.segment(im, gm)
            u_ref, _, st_ref = ref.reduce_noise_tiles(dt, gt, ms, alpha)
            a = ref.stitch(u_ref, im.shape)
            b = s.reduce_noise(im, gm)
            worst = max(worst, (a - b).abs().max().item())
    assert worst <= 0.02, worst


def test_reference_segmentation_and_stitching(ref):
    # the device segmentation and stitching of oracle/refgpu.py are the
    # host loops of cuda/pyCUDANCS/ncs.py:81-98 and :161-169: solving the
    # identity (stitching the input tiles) returns the frame, and the tile
    # origins follow range(0, H + 2, 14) with the last ones moved back
    from oracle import numpy_ref as nr
    for H, W in [(512, 512), (70, 61), (27, 29), (14, 14)]:
        x = torch.rand(2, H, W, device="cuda")
        g = torch.rand(H, W, device="cuda")
        dt, gt = ref.segment(x, g)
        assert torch.equal(ref.stitch(dt, x.shape), x)
        assert dt.shape[0] == 2 * len(range(0, H + 2, 14)) * len(range(0, W + 2, 14))
        assert sorted(set(ref.origins(H))) == nr.tile_origins(H)
