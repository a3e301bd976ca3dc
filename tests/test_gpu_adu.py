"""GPU tests of the preprocessing prologue (ncsb_reduce_noise_adu).

The library converts raw ADU counts with the camera calibration
(python3-6/pyNCS/denoisetools.py:222-224 and :266, matlab/genmaps.m:29-62)
in one device pass before the solve.  It computes d = (ADU - offset) / gain
and gamma = var / gain^2 with IEEE float32 subtraction, division and
multiplication, so it must reproduce bit for bit the solve of photo-electron
frames preprocessed by the same float32 operations elsewhere; against the
FP64 oracle preprocessing (oracle/numpy_ref.py adu_to_photons) the solves
agree to rounding.
"""
import numpy
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ncs(cuda_ok):
    import ncs_b200
    return ncs_b200


def camera(T, H, W, L, seed):
    """Raw frames from the sim's camera model, with L amplifiers whose gains
    differ by level (ADU thresholds 120 and 160)."""
    from ncs_b200 import sim
    rng = numpy.random.default_rng(seed)
    w = sim.make_stack("frame256", T=T, seed=seed, H=H, W=W, chains=3)
    offset, gain0, var0 = sim.camera_maps(H, W, rng)
    gain = numpy.stack([gain0 * (1.0 + 0.15 * k) for k in range(L)]).astype(numpy.float32)
    var = numpy.stack([var0 * (1.0 + 0.3 * k) for k in range(L)]).astype(numpy.float32)
    phot = torch.poisson(torch.as_tensor(w["ideal"], dtype=torch.float32).expand(T, H, W)
                         .contiguous(), generator=torch.Generator().manual_seed(seed))
    adu = (phot * torch.from_numpy(gain0.astype(numpy.float32))
           + torch.from_numpy(numpy.sqrt(var0).astype(numpy.float32)) * torch.randn(
               (T, H, W), generator=torch.Generator().manual_seed(seed + 1))
           + torch.from_numpy(offset.astype(numpy.float32)))
    levels = (120.0, 160.0)[:L - 1]
    return (adu.cuda(), torch.from_numpy(offset.astype(numpy.float32)).cuda(),
            torch.from_numpy(gain).cuda(), torch.from_numpy(var).cuda(), levels, w["mask"])


def torch_prologue(adu, offset, gain, var, levels):
    """The same float32 operations as the library's conversion pass, in torch."""
    lv = torch.zeros(adu.shape, dtype=torch.long, device=adu.device)
    for t in levels:
        lv += (adu >= t).long()
    H, W = adu.shape[1:]
    r = torch.arange(H, device=adu.device).view(1, H, 1)
    c = torch.arange(W, device=adu.device).view(1, 1, W)
    g = gain[lv, r, c]
    v = var[lv, r, c]
    d = (adu - offset) / g
    d = torch.where(d <= 0, torch.full_like(d, 1e-6), d)
    return d.contiguous(), (v / (g * g)).contiguous()


@pytest.mark.parametrize("L", [1, 2, 3])
def test_fused_prologue_is_bitwise_the_two_step_solve(ncs, L):
    adu, off, gain, var, levels, mask = camera(3, 70, 61, L, seed=10 + L)
    s = ncs.Solver(alpha=0.2)
    s.set_otf_mask(mask)
    out, it, st, cost, ev = s.reduce_noise_adu(adu, off, gain, var, levels, tile_stats=True)
    d, g = torch_prologue(adu, off, gain, var, levels)
    ref, rit, rst, rcost, rev = s.reduce_noise(d, g, tile_stats="all")
    assert torch.equal(out, ref) and torch.equal(it, rit) and torch.equal(cost, rcost)
    assert (st == 0).all()


def test_fused_prologue_vs_fp64_oracle_preprocessing(ncs):
    from oracle import numpy_ref as nr
    adu, off, gain, var, levels, mask = camera(2, 48, 48, 2, seed=31)
    s = ncs.Solver(alpha=0.2, epsilon=1e-6)
    s.set_otf_mask(mask)
    out, it, st, cost, ev = s.reduce_noise_adu(adu, off, gain, var, levels, tile_stats=True)
    d, g = nr.adu_to_photons(adu.cpu().numpy(), off.cpu().numpy(), gain.cpu().numpy(),
                             var.cpu().numpy(), levels)
    ref = s.reduce_noise(torch.from_numpy(d.astype(numpy.float32)).cuda(),
                         torch.from_numpy(g.astype(numpy.float32)).cuda())
    # the two preprocessings differ by at most an ulp per pixel; both solves
    # converge to the same optimum
    rel = ((out - ref).abs() / ref.abs().clamp(min=1.0)).max().item()
    assert rel <= 1e-3


def test_adu_errors(ncs):
    adu, off, gain, var, levels, mask = camera(1, 32, 32, 2, seed=5)
    s = ncs.Solver(alpha=0.2)
    s.set_otf_mask(mask)
    with pytest.raises(ValueError):
        s.reduce_noise_adu(adu, off, gain, var, ())            # 2 pairs need 1 threshold
    with pytest.raises(RuntimeError):
        s.reduce_noise_adu(adu, off, gain, var, (float("nan"),))    # non-finite threshold
    # the prologue feeds every solver form: the plain form on raw frames equals
    # the plain form on frames converted with the same FP32 operations
    p = ncs.Solver(alpha=0.2, mode="plain")
    p.set_otf_mask(mask)
    d, g = torch_prologue(adu, off, gain, var, levels)
    assert torch.equal(p.reduce_noise_adu(adu, off, gain, var, levels), p.reduce_noise(d, g))
