"""GPU tests of the normalised single-pixel variant
(ncsb_reduce_noise_normalized) against its FP64 oracle
(oracle/normalized_ref.py): per-pixel final cost within 1e-9 relative of
the exact optimum when run to convergence, the segment centres as output,
replicate-padded borders, per-frame gamma, the iteration cap of the
reference's demos (15), and argument checks.
"""
import numpy
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ncs(cuda_ok):
    import ncs_b200
    return ncs_b200


def data(T, H, W, seed, per_frame=False):
    rng = numpy.random.default_rng(seed)
    ideal = 10 + 60 * numpy.exp(-((numpy.arange(W)[None, :] - W / 2) ** 2 +
                                 (numpy.arange(H)[:, None] - H / 3) ** 2) / 8.0)
    gshape = (T, H, W) if per_frame else (H, W)
    gamma = rng.exponential(15.0, size=gshape) + 0.3
    im = rng.poisson(ideal, size=(T, H, W)) + rng.normal(0, 2.0, size=(T, H, W))
    im = numpy.where(im <= 0, 1e-6, im)
    return im.astype(numpy.float32), gamma.astype(numpy.float32)


@pytest.mark.parametrize("per_frame", [False, True])
def test_converged_pixels_match_the_fp64_optimum(ncs, per_frame):
    from ncs_b200 import otf
    from oracle import normalized_ref as nr
    T, H, W = 2, 9, 11
    im, gam = data(T, H, W, 3, per_frame)
    mask = otf.normalized_mask(0.1, 1.4, 0.7).astype(numpy.float32)
    out, it, st, cost = ncs.reduce_noise_normalized(
        torch.from_numpy(im).cuda(), torch.from_numpy(gam).cuda(), mask, alpha=1.0,
        max_iters=500, tol=1e-9, stats=True)
    out, st, cost = out.cpu().numpy(), st.cpu().numpy(), cost.cpu().numpy()
    # converged: the gradient test, or an FP64 step too small to move u
    assert numpy.isin(st, (0, -5)).all(), numpy.unique(st, return_counts=True)
    m64 = mask.astype(numpy.float64)
    for f in range(T):
        g = gam[f] if per_frame else gam
        ref, fstar = nr.reduce_noise(im[f], g, m64, 1.0)
        gap = (cost[f].ravel() - fstar) / numpy.maximum(numpy.abs(fstar), 1.0)
        assert gap.max() <= 1e-9 and gap.min() >= -1e-9
        assert numpy.abs(out[f] - ref).max() <= 1e-4 * max(1.0, numpy.abs(ref).max())


def test_large_relative_steps_match_the_fp64_optimum(ncs):
    # dead pixels (1e-6) beside bright ones, and hot pixels, with a small gamma:
    # the first steps move u + gamma by far more than the 30 % the line search's
    # series log1p covers, so the library log1p branch runs as well
    from ncs_b200 import otf
    from oracle import normalized_ref as nr
    H, W = 8, 10
    rng = numpy.random.default_rng(11)
    im = rng.poisson(80.0, size=(1, H, W)).astype(numpy.float64)
    im[0, ::3, ::2] = 1e-6
    im[0, 1::4, 1::3] *= 6.0
    im = im.astype(numpy.float32)
    gam = numpy.full((H, W), 0.3, numpy.float32)
    mask = otf.normalized_mask(0.1, 1.4, 0.7).astype(numpy.float32)
    out, it, st, cost = ncs.reduce_noise_normalized(
        torch.from_numpy(im).cuda(), torch.from_numpy(gam).cuda(), mask, alpha=1.0,
        max_iters=500, tol=1e-9, stats=True)
    st, cost = st.cpu().numpy(), cost.cpu().numpy()
    assert numpy.isin(st, (0, -5)).all(), numpy.unique(st, return_counts=True)
    _, fstar = nr.reduce_noise(im[0], gam, mask.astype(numpy.float64), 1.0)
    gap = (cost[0].ravel() - fstar) / numpy.maximum(numpy.abs(fstar), 1.0)
    assert gap.max() <= 1e-9 and gap.min() >= -1e-9


def test_iteration_cap_of_the_reference_demos(ncs):
    from ncs_b200 import otf
    im, gam = data(1, 16, 16, 5)
    mask = otf.normalized_mask()
    out, it, st, cost = ncs.reduce_noise_normalized(
        torch.from_numpy(im).cuda(), torch.from_numpy(gam).cuda(), mask, stats=True)
    it, st = it.cpu().numpy(), st.cpu().numpy()
    assert it.max() <= 15
    assert set(numpy.unique(st)) <= {0, -2, -5}
    assert (out.cpu().numpy() > 0).all()


def test_argument_checks(ncs):
    im = torch.ones((1, 8, 8), device="cuda")
    with pytest.raises(ValueError):
        ncs.reduce_noise_normalized(im, torch.ones((7, 8), device="cuda"), numpy.ones((3, 3)))
    with pytest.raises(ValueError):
        ncs.reduce_noise_normalized(im, torch.ones((8, 8), device="cuda"), numpy.ones((4, 4)))
    with pytest.raises(ValueError):
        ncs.reduce_noise_normalized(im, torch.ones((8, 8), device="cuda"), numpy.ones((3, 3)),
                                    alpha=-1.0)


def test_cost_known_answer_from_calcost(ncs):
    """The kernel's cost at the start u = d for the centre pixel of a 3 x 3
    frame -- whose segment is the whole frame -- equals the value derived by
    hand from calcost.m (tests/test_normalized_cpu.py states the derivation):
    u = d = [[2, 3, 1], [1, 1, 1], [1, 1, 1]], gamma 2, alpha 1/2, mask
    [[1, 2, 1], [1, 1/2, 1], [1, 2, 1]]; within 1e-6 relative."""
    from test_normalized_cpu import KNOWN_COST, KNOWN_MASK, KNOWN_U
    im = torch.tensor([KNOWN_U], dtype=torch.float32, device="cuda")
    gam = torch.full((3, 3), 2.0, dtype=torch.float32, device="cuda")
    out, it, st, cost = ncs.reduce_noise_normalized(im, gam, numpy.array(KNOWN_MASK),
                                                    alpha=0.5, max_iters=0, stats=True)
    assert int(it[0, 1, 1].item()) == 0
    c = float(cost[0, 1, 1].item())
    assert abs(c - KNOWN_COST) <= 1e-6 * abs(KNOWN_COST), (c, KNOWN_COST)
