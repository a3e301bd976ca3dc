"""GPU tests of the learned warm start (libncs_b200.so, ncsb_net_* and
ncsb_reduce_noise_start).

* the network kernels against the FP64 oracle (oracle/warmstart_ref.py):
  forward activations, the full backpropagated gradient of the MSE loss,
  one Adam step, the fused inference kernel (tile and stack mode);
* the solver's proposed-start path: a proposal equal to the photon image, or
  one so bad that every tile falls back, reproduces the plain start bit for
  bit; the converged solution as proposal stops at once;
* training on the GPU lowers the loss, and the trained network lowers the
  L-BFGS iteration count against the solve from the photon image at equal
  accuracy (per-tile cost within 1e-4 relative of the FP64 optimum).
Tolerances are stated per test.
"""
import os

import numpy
import pytest
import torch

from oracle import warmstart_ref as wr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ws(cuda_ok):
    from ncs_b200 import warmstart
    return warmstart


def case(ws, n=12, seed=0):
    rng = numpy.random.default_rng(seed)
    d = rng.uniform(0.0, 80.0, size=(n, 16, 16)).astype(numpy.float32)
    g = rng.exponential(15.0, size=(n, 16, 16)).astype(numpy.float32)
    p = ws.init_params(seed)
    wo, nw, bo, nb = ws.layer_offsets()[3]
    p[wo:wo + nw] = rng.normal(0.0, 0.05, nw)
    p[bo] = 0.1
    for li in range(3):
        wo, nw, bo, nb = ws.layer_offsets()[li]
        p[bo:bo + nb] = rng.normal(0.0, 0.05, nb).astype(numpy.float32)
    target = rng.normal(0.0, 0.5, size=(n, 1, 16, 16)).astype(numpy.float32)
    return p, d, g, target


def test_forward_matches_oracle(ws):
    p, d, g, _ = case(ws)
    net = ws.WarmStartNet(p)
    x, sc = net.features(torch.from_numpy(d).cuda(), torch.from_numpy(g).cuda())
    xo, mu, sd = wr.features(d, g)
    # features: FP32 one-pass moments vs FP64
    assert numpy.allclose(x.cpu().numpy(), xo, rtol=1e-4, atol=1e-4)
    assert numpy.allclose(sc[:, 1].cpu().numpy(), sd, rtol=1e-5)
    acts = net.forward(x)
    ao = wr.forward(p.astype(numpy.float64), x.cpu().numpy().astype(numpy.float64))
    for a, b in zip(acts, ao):
        a = a.cpu().numpy()
        # FP32 accumulation over up to 288 terms: 1e-5 of the layer's scale
        assert numpy.abs(a - b).max() <= 1e-5 * max(1.0, numpy.abs(b).max())


def test_gradient_matches_oracle(ws):
    """The GPU's backpropagated gradient equals the oracle's (which is pinned
    against finite differences and torch autograd on the CPU)."""
    p, d, g, target = case(ws, n=12, seed=4)
    net = ws.WarmStartNet(p)
    x, _ = net.features(torch.from_numpy(d).cuda(), torch.from_numpy(g).cuda())
    x = x.clone()
    loss, grad = net.loss_and_grad(x, torch.from_numpy(target).cuda())
    lo, go = wr.loss_and_grad(p.astype(numpy.float64), x.cpu().numpy().astype(numpy.float64),
                              target.astype(numpy.float64))
    assert abs(loss.item() - lo) <= 1e-5 * lo
    grad = grad.cpu().numpy()
    for wo, nw, bo, nb in ws.layer_offsets():
        for a, b in ((grad[wo:wo + nw], go[wo:wo + nw]), (grad[bo:bo + nb], go[bo:bo + nb])):
            # FP32 sums over 12 x 256 pixels: 1e-4 of the block's largest entry
            assert numpy.abs(a - b).max() <= 1e-4 * numpy.abs(b).max() + 1e-9


def test_adam_step_matches_oracle(ws):
    p, d, g, target = case(ws, n=4, seed=5)
    net = ws.WarmStartNet(p)
    x, _ = net.features(torch.from_numpy(d).cuda(), torch.from_numpy(g).cuda())
    x = x.clone()
    t = torch.from_numpy(target).cuda()
    w, m, v = p.astype(numpy.float64), numpy.zeros(p.size), numpy.zeros(p.size)
    for step in (1, 2, 3):
        _, grad = net.loss_and_grad(x, t)
        gnp = grad.cpu().numpy().astype(numpy.float64)
        w_before = net.params.cpu().numpy().astype(numpy.float64)
        net.adam_step(grad, lr=1e-3)
        w, m, v = wr.adam(w_before, gnp, m, v, step, lr=1e-3)
        assert numpy.abs(net.params.cpu().numpy() - w).max() <= 1e-6


def test_fused_inference_matches_oracle_and_layers(ws):
    p, d, g, _ = case(ws, n=10, seed=6)
    net = ws.WarmStartNet(p)
    dt, gt = torch.from_numpy(d).cuda(), torch.from_numpy(g).cuda()
    u0 = net.propose_tiles(dt, gt).cpu().numpy()
    uo = wr.propose(p.astype(numpy.float64), d, g)
    assert numpy.abs(u0 - uo).max() <= 1e-4 * max(1.0, numpy.abs(uo).max())


def test_stack_inference_equals_tile_inference(ws):
    from ncs_b200 import sim
    w = sim.make_stack("frame256", T=2, seed=11)
    p, _, _, _ = case(ws, seed=7)
    net = ws.WarmStartNet(p)
    us = net.propose_stack(w["images"], w["gamma"])
    d, g = ws.cut_tiles(w["images"], w["gamma"])
    ut = net.propose_tiles(d, g)
    assert torch.equal(us, ut)   # same kernel, only the gather differs
    # per-frame gamma gives the same tiles when every frame has the same map
    us2 = net.propose_stack(w["images"], w["gamma"].expand(2, 256, 256).contiguous())
    assert torch.equal(us, us2)


@pytest.fixture(scope="module")
def stack(cuda_ok):
    from ncs_b200 import sim
    return sim.make_stack("frame256", T=3, seed=21)


def spectral_solver(w, **kw):
    import ncs_b200
    s = ncs_b200.Solver(alpha=w["alpha"], **kw)
    s.set_otf_mask(w["mask"])
    return s


def test_photon_image_proposal_is_bitwise_plain_start(ws, stack):
    s = spectral_solver(stack)
    out0, it0, st0, c0, ev0 = s.reduce_noise(stack["images"], stack["gamma"], tile_stats="all")
    d, _ = ws.cut_tiles(stack["images"], stack["gamma"])
    out1, it1, st1, c1, ev1, fb = s.reduce_noise_from(stack["images"], stack["gamma"], d)
    assert torch.equal(out0, out1) and torch.equal(it0, it1) and torch.equal(c0, c1)
    assert (fb == 0).all()   # equal cost: the proposal is kept


def test_bad_proposal_falls_back_bitwise(ws, stack):
    s = spectral_solver(stack)
    out0, it0, st0, c0, ev0 = s.reduce_noise(stack["images"], stack["gamma"], tile_stats="all")
    d, _ = ws.cut_tiles(stack["images"], stack["gamma"])
    bad = d + 500.0
    out1, it1, st1, c1, ev1, fb = s.reduce_noise_from(stack["images"], stack["gamma"], bad)
    assert (fb == 1).all()
    assert torch.equal(out0, out1) and torch.equal(it0, it1) and torch.equal(st0, st1)
    assert torch.equal(c0, c1)


def test_solution_proposal_stops_immediately(ws, stack):
    s = spectral_solver(stack, epsilon=1e-6)
    d, g = ws.cut_tiles(stack["images"], stack["gamma"])
    ustar, it, st, _ = s.solve_tiles(d, g)
    out, it1, st1, c1, ev1, fb = s.reduce_noise_from(stack["images"], stack["gamma"], ustar)
    assert (fb == 0).all()
    assert (it1 <= 1).all() and (st1 == 0).all()


def test_proposal_path_rejects_other_forms(ws, stack):
    s = spectral_solver(stack, mode="plain")
    d, _ = ws.cut_tiles(stack["images"], stack["gamma"])
    with pytest.raises(RuntimeError):
        s.reduce_noise_from(stack["images"], stack["gamma"], d)


def test_training_lowers_loss(ws):
    d, g, u = ws.training_tiles(12000, seed=500, frames=3)
    net = ws.WarmStartNet(seed=1)
    hist = net.train(d, g, u, epochs=3, batch=1024, lr=2e-3)
    assert hist[-1] < 0.6 * hist[0], hist


def test_trained_network_gains_over_photon_image_start(ws):
    """Held-out stack from the training distribution (seeds outside the
    training range): the trained proposal lowers the mean L-BFGS iteration
    count of the spectral solve, both solves reach the FP64 optimum within
    1e-4 relative cost per tile, and the proposal's own cost is lower than
    the photon image's on most tiles."""
    from oracle import numpy_ref as nr
    if os.path.exists(ws.DEFAULT_WEIGHTS):
        net = ws.WarmStartNet.load()
    else:
        d, g, u = ws.training_tiles(40000, seed=1000, frames=3)
        net = ws.WarmStartNet(seed=0)
        net.train(d, g, u, epochs=6, batch=1024)
    w = ws.simulate(987654, "cuda", H=512, W=512, frames=2)
    s = spectral_solver(w)
    out0, it0, st0, c0, _ = s.reduce_noise(w["images"], w["gamma"], tile_stats="all")
    u0 = net.propose_stack(w["images"], w["gamma"])
    out1, it1, st1, c1, _, fb = s.reduce_noise_from(w["images"], w["gamma"], u0)
    it0, it1 = it0.float().mean().item(), it1.float().mean().item()
    assert it1 < 0.9 * it0, (it0, it1)
    assert fb.float().mean().item() < 0.5
    # accuracy of both against the FP64 optimum on a sample of tiles
    d, g = ws.cut_tiles(w["images"], w["gamma"])
    idx = numpy.arange(0, d.shape[0], max(1, d.shape[0] // 48))
    ms = numpy.fft.fftshift(w["mask"]).astype(numpy.float64)
    dn, gn = d.cpu().numpy()[idx], g.cpu().numpy()[idx]
    _, fstar, _ = nr.newton_solve(dn, gn, ms, w["alpha"])
    for c in (c0, c1):
        gap = nr.rel_cost_gap(c.cpu().numpy()[idx], fstar)
        assert gap.max() <= 1e-4
