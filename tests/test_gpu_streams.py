"""GPU tests of launches on a caller's stream.

Every entry takes ``stream=``.  The wrappers make contiguous copies and
allocate outputs on the current stream, so on another stream the launch
must wait for that work, and those tensors must not be reused by the
caching allocator before the launch is done (ncs_b200.ncs.launch_stream).
Inputs here are non-contiguous views, so the copies exist, and the current
stream is kept busy with allocations and writes while the side stream runs.
"""
import pytest
import torch

from conftest import create_otf_mask_shifted

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ncs(cuda_ok):
    import ncs_b200
    return ncs_b200


def strided(x):
    """The same values as a non-contiguous view (last two axes transposed
    in memory)."""
    return x.transpose(-1, -2).contiguous().transpose(-1, -2)


def churn():
    # allocations and writes on the current stream while the side stream runs
    for _ in range(4):
        t = torch.empty(8 << 20, device="cuda")
        t.fill_(float("nan"))
        del t


def test_side_stream_with_copied_inputs(ncs):
    g = torch.Generator(device="cuda").manual_seed(11)
    im = 5.0 + 50.0 * torch.rand((3, 64, 70), device="cuda", generator=g)
    gam = 2.0 + 2.0 * torch.rand((64, 70), device="cuda", generator=g)
    s = ncs.Solver(alpha=0.2)
    s.set_otf_mask_shifted(create_otf_mask_shifted())
    ref = s.reduce_noise(im, gam)
    ref_t = s.solve_tiles(im[:, :16, :16].contiguous(), gam[None, :16, :16].expand(3, 16, 16)
                          .contiguous())[0]
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    out = s.reduce_noise(strided(im), strided(gam), stream=side)
    tiles = s.solve_tiles(strided(im[:, :16, :16]), strided(gam[None, :16, :16].expand(3, 16, 16)),
                          stream=side)[0]
    churn()
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    assert torch.equal(tiles, ref_t)


def test_side_stream_raw_counts(ncs):
    g = torch.Generator(device="cuda").manual_seed(12)
    off = 100.0 + torch.rand((48, 40), device="cuda", generator=g)
    gain = 2.0 + 0.2 * torch.rand((48, 40), device="cuda", generator=g)
    var = 40.0 + 20.0 * torch.rand((48, 40), device="cuda", generator=g)
    raw = (off + gain * (10.0 + 40.0 * torch.rand((2, 48, 40), device="cuda", generator=g))
           ).round().to(torch.uint16)
    s = ncs.Solver(alpha=0.2)
    s.set_otf_mask_shifted(create_otf_mask_shifted())
    ref = s.reduce_noise_adu(raw, off, gain, var)
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    out = s.reduce_noise_adu(strided(raw), strided(off), strided(gain), strided(var), stream=side)
    churn()
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
