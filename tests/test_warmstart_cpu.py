"""CPU checks of the warm-start network's oracle and host logic (no GPU).

The FP64 oracle (oracle/warmstart_ref.py) is the checker of the CUDA
network kernels, so it is pinned first: its backpropagated gradient against
central finite differences and against torch autograd (FP64, CPU), its
forward pass against torch's conv2d.  Host logic: the training-data tile
cutter against the pinned segmentation oracle (oracle/numpy_ref.py), and the
parameter layout against the library's count.
"""
import numpy
import pytest
import torch

from oracle import warmstart_ref as wr


def random_case(n=2, seed=0, scale=1.0):
    rng = numpy.random.default_rng(seed)
    d = rng.uniform(0.0, 60.0, size=(n, 16, 16))
    g = rng.exponential(15.0, size=(n, 16, 16))
    from ncs_b200 import warmstart
    p = warmstart.init_params(seed).astype(numpy.float64)
    # a non-zero last layer so every layer receives gradient
    wo, nw, bo, nb = warmstart.layer_offsets()[3]
    p[wo:wo + nw] = rng.normal(0.0, 0.05 * scale, nw)
    p[bo] = 0.1
    for li in range(3):
        wo, nw, bo, nb = warmstart.layer_offsets()[li]
        p[bo:bo + nb] = rng.normal(0.0, 0.05, nb)
    x, mu, sd = wr.features(d, g)
    target = rng.normal(0.0, 0.5, size=(n, 1, 16, 16))
    return p, x, target, d, g


def torch_reference(p, x, target):
    """Loss and packed gradient through torch.nn.functional.conv2d in FP64."""
    ws = []
    for w, b in wr.unpack(p):
        cin, _, cout = w.shape
        wt = torch.tensor(w.reshape(cin, 3, 3, cout).transpose(3, 0, 1, 2).copy(),
                          requires_grad=True)
        bt = torch.tensor(b.copy(), requires_grad=True)
        ws.append((wt, bt))
    cur = torch.tensor(x)
    for li, ((wt, bt), (_, _, relu)) in enumerate(zip(ws, wr.LAYERS)):
        cur = torch.nn.functional.conv2d(cur, wt, bt, padding=1)
        if relu:
            cur = torch.relu(cur)
    loss = torch.mean((cur - torch.tensor(target)) ** 2)
    loss.backward()
    grads = []
    for wt, bt in ws:
        gw = wt.grad.numpy()  # [co, ci, 3, 3] -> [ci, 9, co]
        grads.append((gw.transpose(1, 2, 3, 0).reshape(gw.shape[1], 9, gw.shape[0]),
                       bt.grad.numpy()))
    return float(loss.detach()), wr.pack(grads), cur.detach().numpy()


def test_oracle_matches_torch_autograd():
    p, x, target, _, _ = random_case()
    loss, grad = wr.loss_and_grad(p, x, target)
    tloss, tgrad, ty = torch_reference(p, x, target)
    assert numpy.allclose(wr.forward(p, x)[3], ty, rtol=1e-12, atol=1e-12)
    assert abs(loss - tloss) <= 1e-12 * max(1.0, abs(tloss))
    assert numpy.allclose(grad, tgrad, rtol=1e-10, atol=1e-14)


def test_oracle_gradient_vs_finite_differences():
    p, x, target, _, _ = random_case(seed=3)
    _, grad = wr.loss_and_grad(p, x, target)
    rng = numpy.random.default_rng(7)
    from ncs_b200 import warmstart
    idx = []
    for wo, nw, bo, nb in warmstart.layer_offsets():   # weights and biases of every layer
        idx += list(rng.choice(numpy.arange(wo, wo + nw), 6, replace=False)) + [bo]
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (wr.loss_and_grad(pp, x, target)[0] - wr.loss_and_grad(pm, x, target)[0]) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-6 * max(1.0, abs(grad[i])) + 1e-9, (i, fd, grad[i])


def test_oracle_adam_first_step_is_signed_lr():
    w = numpy.zeros(5)
    g = numpy.array([1.0, -2.0, 0.5, 3.0, -0.1])
    w1, m, v = wr.adam(w, g, numpy.zeros(5), numpy.zeros(5), 1, lr=0.01, eps=0.0)
    assert numpy.allclose(w1, -0.01 * numpy.sign(g))


def test_proposal_clamp_keeps_start_feasible():
    p, x, target, d, g = random_case(scale=200.0)   # a wild last layer
    u0 = wr.propose(p, d, g)
    assert (u0 + g >= wr.START_FRAC * numpy.maximum(d + g, 1e-3) - 1e-12).all()


def test_e4m3_rounding_matches_torch_float8():
    """The oracle's E4M3 rounding (the checker of the tensor-core inference's
    FP8 form) equals torch's float8_e4m3fn conversion: ties to even, the
    subnormal spacing 2^-9 below 2^-6, saturation at +-448."""
    rng = numpy.random.default_rng(3)
    x = rng.normal(0.0, 1.0, 50000) * 10.0 ** rng.uniform(-4.0, 3.0, 50000)
    edge = [0.0, -0.0, 448.0, -448.0, 464.0, 1e4, -1e4, 2.0 ** -9, 2.0 ** -10,
            3 * 2.0 ** -11, 2.0 ** -6, 1.0625, 1.1875, 15.5, 240.0, 248.0]
    x = numpy.concatenate([x, edge]).astype(numpy.float32).astype(numpy.float64)
    ref = torch.from_numpy(numpy.clip(x, -448.0, 448.0).astype(numpy.float32)).to(
        torch.float8_e4m3fn).to(torch.float64).numpy()
    assert numpy.array_equal(wr.round_e4m3(x), ref)


def test_fp8_forward_reduces_to_the_network_without_rounding(monkeypatch):
    """forward_fp8 with the rounding switched off is the FP64 network: its
    scales cancel exactly."""
    p, x, target, d, g = random_case(seed=4)
    monkeypatch.setattr(wr, "round_e4m3", lambda v: numpy.asarray(v, dtype=numpy.float64))
    assert numpy.allclose(wr.forward_fp8(p, x), wr.forward(p, x)[3], rtol=1e-12, atol=1e-12)


def test_parameter_layout():
    from ncs_b200 import _lib, warmstart
    assert warmstart.N_PARAMS == 19393
    assert _lib.load().ncsb_net_param_count() == warmstart.N_PARAMS
    off = warmstart.layer_offsets()
    assert off[0][0] == 0 and off[-1][2] + off[-1][3] == warmstart.N_PARAMS
    # the library's float4 weight reads need 16-byte aligned weight blocks
    assert all(wo % 4 == 0 for wo, _, _, _ in off)
    p = warmstart.init_params(0)
    assert p.dtype == numpy.float32 and not p[off[3][0]:].any()   # untrained net proposes d


@pytest.mark.parametrize("hw", [(14, 14), (37, 53), (256, 256)])
def test_cut_tiles_matches_segmentation_oracle(hw):
    from ncs_b200 import warmstart
    from oracle import numpy_ref as nr
    H, W = hw
    rng = numpy.random.default_rng(H * W)
    im = rng.uniform(0, 100, size=(2, H, W)).astype(numpy.float32)
    ga = rng.uniform(1, 5, size=(H, W)).astype(numpy.float32)
    d, g = warmstart.cut_tiles(torch.from_numpy(im), torch.from_numpy(ga))
    td, tg, meta = nr.segment(im, ga)
    assert numpy.array_equal(d.numpy(), td.astype(numpy.float32))
    assert numpy.array_equal(g.numpy(), tg.astype(numpy.float32))
