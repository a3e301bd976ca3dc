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


def integer_counts(adu, dtype):
    """The camera's counts as stored: rounded and clipped to the type's range."""
    hi = 255.0 if dtype == torch.uint8 else 65535.0
    return adu.round().clamp(0.0, hi).to(dtype)


@pytest.mark.parametrize("dtype", [torch.uint16, torch.uint8])
@pytest.mark.parametrize("W,L", [(64, 1), (61, 1), (64, 2)])
def test_integer_counts_equal_the_same_counts_in_float32(ncs, dtype, W, L):
    # W = 64 takes the 4-wide path (one pair), W = 61 and two pairs the scalar one
    adu, off, gain, var, levels, mask = camera(3, 40, W, L, seed=50 + W + L)
    raw = integer_counts(adu, dtype)
    s = ncs.Solver(alpha=0.2)
    s.set_otf_mask(mask)
    out = s.reduce_noise_adu(raw, off, gain, var, levels)
    ref = s.reduce_noise_adu(raw.float(), off, gain, var, levels)
    assert torch.equal(out, ref)
    d, g = torch_prologue(raw.float(), off, gain, var, levels)
    assert torch.equal(out, s.reduce_noise(d, g))


@pytest.mark.parametrize("dtype", [torch.float32, torch.uint16, torch.uint8])
@pytest.mark.parametrize("L", [1, 3])
def test_host_raw_pipeline_equals_the_device_entry(ncs, dtype, L):
    adu, off, gain, var, levels, mask = camera(7, 48, 52, L, seed=70 + L)
    raw = adu if dtype == torch.float32 else integer_counts(adu, dtype)
    s = ncs.Solver(alpha=0.2)
    s.set_otf_mask(mask)
    ref = s.reduce_noise_adu(raw, off, gain, var, levels).cpu()
    h_raw = raw.cpu()
    # pageable input, default chunks; page-locked input and output, 1-frame
    # chunks over 3 streams (the last chunk is reused by stream 0 twice)
    assert torch.equal(s.reduce_noise_adu_host(h_raw, off, gain, var, levels), ref)
    pinned_out = torch.empty(ref.shape, dtype=torch.float32).pin_memory()
    got = s.reduce_noise_adu_host(h_raw.pin_memory(), off, gain, var, levels, out=pinned_out,
                                  chunk_frames=1, n_streams=3)
    assert got is pinned_out and torch.equal(got, ref)
    # numpy input
    assert torch.equal(s.reduce_noise_adu_host(h_raw.numpy(), off, gain, var, levels), ref)


def test_unaligned_maps_and_frames_take_the_scalar_path(ncs):
    # views 4 (maps) and 2 (uint16 frames) bytes past an allocation's start
    # cannot be read 16 bytes at a time; the host sees it and the kernel reads
    # them one element at a time, with the same result
    adu, off, gain, var, levels, mask = camera(2, 32, 64, 1, seed=90)
    raw = integer_counts(adu, torch.uint16)
    s = ncs.Solver(alpha=0.2)
    s.set_otf_mask(mask)
    ref = s.reduce_noise_adu(raw, off, gain, var, levels)

    def shifted(x):
        buf = torch.empty(x.numel() + 1, dtype=x.dtype, device=x.device)
        buf[1:] = x.reshape(-1)
        return buf[1:].view(x.shape)
    u_off, u_gain, u_var, u_raw = shifted(off), shifted(gain), shifted(var), shifted(raw)
    assert u_off.data_ptr() % 16 and u_raw.data_ptr() % 8
    assert torch.equal(s.reduce_noise_adu(u_raw, u_off, u_gain, u_var, levels), ref)
    assert torch.equal(s.reduce_noise_adu(raw, u_off, gain, var, levels), ref)


def test_adu_type_errors(ncs):
    adu, off, gain, var, levels, mask = camera(1, 32, 32, 1, seed=6)
    s = ncs.Solver(alpha=0.2)
    s.set_otf_mask(mask)
    with pytest.raises(TypeError):
        s.reduce_noise_adu(adu.to(torch.int32), off, gain, var, levels)
    with pytest.raises(TypeError):
        s.reduce_noise_adu_host(adu, off, gain, var, levels)          # device frames
    with pytest.raises(TypeError):
        s.reduce_noise_adu_host(adu.cpu().double(), off, gain, var, levels)


def test_more_frames_than_one_grid_dimension(ncs):
    # 530,000 frames: the conversion grid's frame dimension (chunks of 8
    # frames) stops at 65,535 and strides over the rest; the solve covers
    # every frame
    T, H, W = 530000, 16, 16
    g = torch.Generator(device="cuda").manual_seed(3)
    off = torch.full((H, W), 100.0, device="cuda")
    gain = 2.0 + 0.1 * torch.rand((H, W), device="cuda", generator=g)
    var = 50.0 + torch.rand((H, W), device="cuda", generator=g)
    phot = 20.0 + 10.0 * torch.rand((T, H, W), device="cuda", generator=g)
    raw = (phot * gain + off).round().to(torch.uint16)
    s = ncs.Solver(alpha=0.2, max_iters=5)
    from conftest import create_otf_mask_shifted
    s.set_otf_mask_shifted(create_otf_mask_shifted())
    out = s.reduce_noise_adu(raw, off, gain, var)
    d = (raw.float() - off) / gain
    d = torch.where(d <= 0, torch.full_like(d, 1e-6), d)
    ref = s.reduce_noise(d, var / (gain * gain))
    assert torch.equal(out, ref)
