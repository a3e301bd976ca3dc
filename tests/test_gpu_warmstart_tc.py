"""GPU tests of the tensor-core inference of the warm-start network
(ncsb_net_infer_stack_tc / ncsb_net_infer_tiles_tc and their _fp8 forms,
tcgen05 with BF16 or E4M3 operands and FP32 accumulation in tensor memory).

BF16, against the FP64 network oracle (oracle/warmstart_ref.py) and the FP32
SIMT inference: proposals agree to BF16 rounding -- max 0.1 and mean 0.005 of
the tile's scale s.  E4M3, against the oracle's E4M3 restatement
(warmstart_ref.propose_fp8: the same scales and roundings, exact
accumulation): mean 1e-4 of s, max 2e-3 on random tiles; on simulated frames
(1,083 tiles) single pixels reach 0.05 of s, because the FP32 accumulation
order can move an activation across an E4M3 rounding boundary, so the bound
there is 0.1 with at most 1e-3 of the pixels above 1e-3; against the FP64 network,
mean 0.05 of s and a maximum of 0.3 of s on random tiles and 1.0 on
simulated frames (single pixels; the oracle's own E4M3 restatement reaches
0.73 there).  In both forms no tensor-core wait times out,
stack and tile modes agree bit for bit, and the spectral solve from the
tensor-core proposals keeps the warm start's iteration gain at the accuracy
of the solve without it.
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


@pytest.mark.parametrize("trained", [True, False])
def test_fp8_inference_matches_fp8_oracle(ws, trained):
    rng = numpy.random.default_rng(12)
    if trained:
        net = ws.WarmStartNet.load()
    else:
        p = ws.init_params(5)
        wo, nw, bo, nb = ws.layer_offsets()[3]
        p[wo:wo + nw] = rng.normal(0, 0.05, nw)
        net = ws.WarmStartNet(p)
    d = rng.uniform(0.0, 90.0, size=(41, 16, 16)).astype(numpy.float32)
    g = rng.exponential(15.0, size=(41, 16, 16)).astype(numpy.float32)
    u, st = net.propose_tiles_tc(torch.from_numpy(d).cuda(), torch.from_numpy(g).cuda(),
                                 fp8=True)
    assert int(st.item()) == 0
    params = net.params.cpu().numpy().astype(numpy.float64)
    _, _, sd = wr.features(d, g)
    u = u.cpu().numpy()
    e8 = numpy.abs(u - wr.propose_fp8(params, d, g)) / sd[:, None, None]
    assert e8.max() <= 2e-3 and e8.mean() <= 1e-4, (e8.max(), e8.mean())
    e64 = numpy.abs(u - wr.propose(params, d, g)) / sd[:, None, None]
    assert e64.max() <= 0.3 and e64.mean() <= 0.05, (e64.max(), e64.mean())


@pytest.mark.parametrize("fp8", [False, True])
def test_tc_stack_equals_tiles_and_solve_gain(ws, fp8):
    import ncs_b200
    from ncs_b200 import sim
    w = sim.make_stack("frame256", T=3, seed=5)
    net = ws.WarmStartNet.load()
    us, st = net.propose_stack_tc(w["images"], w["gamma"], fp8=fp8)
    d, g = ws.cut_tiles(w["images"], w["gamma"])
    ut, st2 = net.propose_tiles_tc(d, g, fp8=fp8)
    assert int(st.item()) == 0 and int(st2.item()) == 0
    assert torch.equal(us, ut)
    u32 = net.propose_stack(w["images"], w["gamma"])
    _, sc = net.features(d, g)
    e = (us - u32).abs() / sc[:, 1].view(-1, 1, 1)
    if fp8:
        assert e.max().item() <= 1.0 and e.mean().item() <= 0.05
        dn, gn = d.cpu().numpy().astype(numpy.float64), g.cpu().numpy().astype(numpy.float64)
        ref = wr.propose_fp8(net.params.cpu().numpy().astype(numpy.float64), dn, gn)
        e8 = numpy.abs(us.cpu().numpy() - ref) / sc[:, 1].cpu().numpy()[:, None, None]
        assert e8.max() <= 0.1 and e8.mean() <= 1e-4, (e8.max(), e8.mean())
        assert (e8 > 1e-3).mean() <= 1e-3, (e8 > 1e-3).mean()
    else:
        assert e.max().item() <= 0.1 and e.mean().item() <= 0.005
    s = ncs_b200.Solver(alpha=w["alpha"])
    s.set_otf_mask(w["mask"])
    _, it0, st0, c0, _ = s.reduce_noise(w["images"], w["gamma"], tile_stats="all")
    _, it1, st1, c1, _, fb = s.reduce_noise_from(w["images"], w["gamma"], us)
    assert (st1 == 0).all()
    assert it1.float().mean().item() <= it0.float().mean().item() - 0.5
    rel = ((c1 - c0).abs() / c0.abs().clamp(min=1.0)).max().item()
    assert rel <= 1e-6   # both converge to the same per-tile optimum


def test_fp8_many_tiles_per_slot(ws):
    """Each slot of the E4M3 kernel processes several tiles in turn (20 frames
    of 256 x 256: about eight per slot), so its activation copies are reused
    with their zero rows and columns: sampled tiles match the oracle's E4M3
    restatement at every position in the order they ran."""
    from ncs_b200 import sim
    w = sim.make_stack("frame256", T=20, seed=9)
    net = ws.WarmStartNet.load()
    u, st = net.propose_stack_tc(w["images"], w["gamma"], fp8=True)
    assert int(st.item()) == 0
    d, g = ws.cut_tiles(w["images"], w["gamma"])
    n = d.shape[0]
    idx = numpy.unique(numpy.concatenate([numpy.arange(0, n, 97), [n - 1]]))
    dn = d.cpu().numpy()[idx].astype(numpy.float64)
    gn = g.cpu().numpy()[idx].astype(numpy.float64)
    ref = wr.propose_fp8(net.params.cpu().numpy().astype(numpy.float64), dn, gn)
    _, _, sd = wr.features(dn, gn)
    e8 = numpy.abs(u.cpu().numpy()[idx] - ref) / sd[:, None, None]
    assert e8.max() <= 0.1 and e8.mean() <= 1e-4, (e8.max(), e8.mean())


def test_fp8_saturating_inputs_stay_finite_and_feasible(ws):
    """Tiles far outside the training range (a hot pixel at 1e5 photons, a
    near-empty tile, a huge gamma, a tile of 1e4..5e4 photons) push features
    and activations beyond E4M3's range: the kernel saturates them as the
    oracle's restatement does, the proposals stay finite and feasible, and the
    solve from them ends at the photon-image solve's cost."""
    import ncs_b200
    from oracle import numpy_ref as nr
    rng = numpy.random.default_rng(21)
    d = rng.uniform(5.0, 30.0, size=(6, 16, 16)).astype(numpy.float32)
    g = rng.exponential(10.0, size=(6, 16, 16)).astype(numpy.float32)
    d[0, 7, 7] = 1.0e5                                 # one hot pixel
    d[1] = 1.0e-6                                      # an empty tile
    g[2] *= 1.0e4                                      # a huge read-noise variance
    d[3] = rng.uniform(1.0e4, 5.0e4, size=(16, 16))    # a tile of bright pixels
    net = ws.WarmStartNet.load()
    dt, gt = torch.from_numpy(d).cuda(), torch.from_numpy(g).cuda()
    u0, st = net.propose_tiles_tc(dt, gt, fp8=True)
    assert int(st.item()) == 0
    u = u0.cpu().numpy().astype(numpy.float64)
    dd, gg = d.astype(numpy.float64), g.astype(numpy.float64)
    assert numpy.isfinite(u).all()
    floor = wr.START_FRAC * numpy.maximum(dd + gg, 1e-3)
    assert (u + gg >= floor * (1.0 - 1e-5) - 1e-6 * (1.0 + gg)).all()
    ref = wr.propose_fp8(net.params.cpu().numpy().astype(numpy.float64), dd, gg)
    _, _, sd = wr.features(dd, gg)
    assert (numpy.abs(u - ref) / sd[:, None, None]).mean() <= 1e-3
    mask = numpy.fft.fftshift(numpy.full((16, 16), 0.5))
    s = ncs_b200.Solver(alpha=0.2)
    s.set_otf_mask(mask)
    u_cold, _, _, _ = s.solve_tiles(dt, gt)
    u_warm, _, _, _ = s.solve_tiles(dt, gt, u0=u0)
    ms = numpy.fft.ifftshift(mask)
    f_cold = nr.cost(u_cold.cpu().numpy().astype(numpy.float64), dd, gg, ms, 0.2)
    f_warm = nr.cost(u_warm.cpu().numpy().astype(numpy.float64), dd, gg, ms, 0.2)
    assert (numpy.abs(f_warm - f_cold) / numpy.maximum(numpy.abs(f_cold), 1.0) <= 1e-5).all()
