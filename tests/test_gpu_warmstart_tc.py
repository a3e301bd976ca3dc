"""GPU tests of the tensor-core inference of the warm-start network
(ncsb_net_infer_stack_tc / ncsb_net_infer_tiles_tc, tcgen05 with BF16
operands and FP32 accumulation in tensor memory).

Against the FP64 network oracle (oracle/warmstart_ref.py) and the FP32 SIMT
inference: proposals agree to BF16 rounding -- max 0.1 and mean 0.005 of the
tile's scale s -- no tensor-core wait times out, stack and tile modes agree
bit for bit, and the spectral solve from the tensor-core proposals keeps the
warm start's iteration gain at the accuracy of the solve without it.
"""
import numpy
import pytest
import torch

from oracle import warmstart_ref as wr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ws(cuda_ok):
    from ncs_b200 import warmstart
    return warmstart


@pytest.mark.parametrize("trained", [True, False])
def test_tc_inference_matches_oracle(ws, trained):
    rng = numpy.random.default_rng(11)
    if trained:
        net = ws.WarmStartNet.load()
    else:
        p = ws.init_params(4)
        wo, nw, bo, nb = ws.layer_offsets()[3]
        p[wo:wo + nw] = rng.normal(0, 0.05, nw)
        net = ws.WarmStartNet(p)
    d = rng.uniform(0.0, 90.0, size=(37, 16, 16)).astype(numpy.float32)
    g = rng.exponential(15.0, size=(37, 16, 16)).astype(numpy.float32)
    u, st = net.propose_tiles_tc(torch.from_numpy(d).cuda(), torch.from_numpy(g).cuda())
    assert int(st.item()) == 0
    ref = wr.propose(net.params.cpu().numpy().astype(numpy.float64), d, g)
    _, _, sd = wr.features(d, g)
    err = numpy.abs(u.cpu().numpy() - ref) / sd[:, None, None]
    assert err.max() <= 0.1 and err.mean() <= 0.005


def test_tc_stack_equals_tiles_and_solve_gain(ws):
    import ncs_b200
    from ncs_b200 import sim
    w = sim.make_stack("frame256", T=3, seed=5)
    net = ws.WarmStartNet.load()
    us, st = net.propose_stack_tc(w["images"], w["gamma"])
    d, g = ws.cut_tiles(w["images"], w["gamma"])
    ut, st2 = net.propose_tiles_tc(d, g)
    assert int(st.item()) == 0 and int(st2.item()) == 0
    assert torch.equal(us, ut)
    u32 = net.propose_stack(w["images"], w["gamma"])
    _, sc = net.features(d, g)
    e = (us - u32).abs() / sc[:, 1].view(-1, 1, 1)
    assert e.max().item() <= 0.1 and e.mean().item() <= 0.005
    s = ncs_b200.Solver(alpha=w["alpha"])
    s.set_otf_mask(w["mask"])
    _, it0, st0, c0, _ = s.reduce_noise(w["images"], w["gamma"], tile_stats="all")
    _, it1, st1, c1, _, fb = s.reduce_noise_from(w["images"], w["gamma"], us)
    assert (st1 == 0).all()
    assert it1.float().mean().item() <= it0.float().mean().item() - 0.5
    rel = ((c1 - c0).abs() / c0.abs().clamp(min=1.0)).max().item()
    assert rel <= 1e-6   # both converge to the same per-tile optimum
