"""FP64 numpy restatement of the warm-start network (test infrastructure).

Only the tests use this module, as the checker of the CUDA kernels in
ncs_b200/csrc/ncs_net.cu (forward, weight and input gradients, Adam, fused
inference).  The network has no counterpart in the reference
(HuanglabPurdue/NCS starts every solve at u = d, clib/pyCNCS/ncs.c:548-551);
what this file restates is the definition the library documents
(include/ncs_b200.h, "learned warm start"): features, four 3x3 zero-padded
convolutions 2 -> 32 -> 32 -> 32 -> 1 with ReLU after the first three, the
proposal u0 = d + s y with its feasibility clamp, the MSE loss, its
gradient by plain backpropagation and one Adam step (Kingma & Ba, 2015).
This restatement is itself checked against central finite differences and
against torch autograd in FP64 on the CPU (tests/test_warmstart_cpu.py).

Weight layout as in the library: wt[ci][tap][co] with tap = 3 ky + kx,
kernel offset (ky - 1, kx - 1); parameters packed w1, b1, w2, b2, w3, b3, w4, b4.
"""
import numpy

C = 32
LAYERS = ((2, C, True), (C, C, True), (C, C, True), (C, 1, False))
START_FRAC = 0.05


def unpack(params):
    p = numpy.asarray(params, dtype=numpy.float64)
    out, o = [], 0
    for cin, cout, _ in LAYERS:
        nw = cin * 9 * cout
        out.append((p[o:o + nw].reshape(cin, 9, cout), p[o + nw:o + nw + cout]))
        o += nw + cout
    assert o == p.size, "parameter count"
    return out


def pack(grads):
    return numpy.concatenate([numpy.concatenate([w.ravel(), b.ravel()]) for w, b in grads])


def features(d, gamma):
    """x [n, 2, 16, 16], mu [n], s [n] (s = population std + 1)."""
    d = numpy.asarray(d, dtype=numpy.float64).reshape(-1, 16, 16)
    g = numpy.asarray(gamma, dtype=numpy.float64).reshape(-1, 16, 16)
    mu = d.mean(axis=(1, 2))
    sd = numpy.sqrt(numpy.maximum((d * d).mean(axis=(1, 2)) - mu * mu, 0.0)) + 1.0
    x0 = (d - mu[:, None, None]) / sd[:, None, None]
    x1 = numpy.sqrt(numpy.maximum(d, 0.0) + numpy.maximum(g, 0.0)) / sd[:, None, None]
    return numpy.stack([x0, x1], axis=1), mu, sd


def _shifted(x, ky, kx):
    """x[..., r + ky - 1, c + kx - 1] with zeros outside the tile."""
    pad = numpy.pad(x, [(0, 0)] * (x.ndim - 2) + [(1, 1), (1, 1)])
    return pad[..., ky:ky + 16, kx:kx + 16]


def conv(x, w, b):
    """y[n, co] = b[co] + sum_ci,tap w[ci, tap, co] x[n, ci](p + off(tap))."""
    n = x.shape[0]
    y = numpy.broadcast_to(b[None, :, None, None], (n, w.shape[2], 16, 16)).copy()
    for tap in range(9):
        xs = _shifted(x, tap // 3, tap % 3)                # [n, ci, 16, 16]
        y += numpy.einsum("nipq,io->nopq", xs, w[:, tap, :])
    return y


def conv_wgrad(x, dy):
    """(dw [ci, 9, co], db [co]) of conv for upstream gradient dy."""
    dw = numpy.stack([numpy.einsum("nipq,nopq->io", _shifted(x, t // 3, t % 3), dy)
                      for t in range(9)], axis=1)
    return dw, dy.sum(axis=(0, 2, 3))


def conv_xgrad(dy, w):
    """dx[n, ci](p) = sum_co,tap w[ci, tap, co] dy[n, co](p - off(tap))."""
    n = dy.shape[0]
    dx = numpy.zeros((n, w.shape[0], 16, 16))
    for tap in range(9):
        ky, kx = tap // 3, tap % 3
        dx += numpy.einsum("nopq,io->nipq", _shifted(dy, 2 - ky, 2 - kx), w[:, tap, :])
    return dx


def forward(params, x):
    """Activations [a1, a2, a3, y] (post-ReLU for the first three)."""
    acts, cur = [], x
    for (w, b), (_, _, relu) in zip(unpack(params), LAYERS):
        z = conv(cur, w, b)
        cur = numpy.maximum(z, 0.0) if relu else z
        acts.append(cur)
    return acts


def propose(params, d, gamma):
    """Proposal u0 [n, 16, 16] (the library's inference, in FP64)."""
    x, mu, sd = features(d, gamma)
    y = forward(params, x)[3][:, 0]
    d = numpy.asarray(d, dtype=numpy.float64).reshape(-1, 16, 16)
    g = numpy.asarray(gamma, dtype=numpy.float64).reshape(-1, 16, 16)
    lo = START_FRAC * numpy.maximum(d + g, 1e-3) - g
    return numpy.maximum(d + sd[:, None, None] * y, lo)


def round_e4m3(x):
    """Round to the nearest E4M3 value (OCP FP8: 1 sign, 4 exponent bits with
    bias 7, 3 mantissa bits, no infinities), ties to even, saturating at
    +-448: the spacing is 2^(e-3) for |x| in [2^e, 2^(e+1)), e >= -6, and
    2^-9 below 2^-6 (subnormals)."""
    x = numpy.clip(numpy.asarray(x, dtype=numpy.float64), -448.0, 448.0)
    a = numpy.abs(x)
    e = numpy.floor(numpy.log2(numpy.where(a > 0, a, 1.0)))
    q = numpy.exp2(numpy.maximum(e, -6.0) - 3.0)
    return numpy.clip(numpy.rint(x / q) * q, -448.0, 448.0)


# E4M3 inference: layer l's input is multiplied by IN_SCALE_FP8[l] before
# rounding; each output column's weights are divided by max|w| / 448
IN_SCALE_FP8 = (8.0, 4.0, 4.0, 4.0)


def forward_fp8(params, x):
    """Output of the network with E4M3 operands: inputs and weights rounded
    after their scaling, products accumulated exactly (FP64 here), scales
    undone before the bias (ncs_b200/csrc/ncs_net_tc.cu, E4M3 form)."""
    cur = numpy.asarray(x, dtype=numpy.float64)
    for li, ((w, b), (_, _, relu)) in enumerate(zip(unpack(params), LAYERS)):
        mx = numpy.abs(w).max(axis=(0, 1))
        sw = numpy.where(mx > 0, mx / 448.0, 1.0)
        wq = round_e4m3(w / sw[None, None, :]) * sw[None, None, :]
        xq = round_e4m3(cur * IN_SCALE_FP8[li]) / IN_SCALE_FP8[li]
        z = conv(xq, wq, b)
        cur = numpy.maximum(z, 0.0) if relu else z
    return cur


def propose_fp8(params, d, gamma):
    """Proposal u0 [n, 16, 16] of the E4M3 tensor-core inference."""
    x, mu, sd = features(d, gamma)
    y = forward_fp8(params, x)[:, 0]
    d = numpy.asarray(d, dtype=numpy.float64).reshape(-1, 16, 16)
    g = numpy.asarray(gamma, dtype=numpy.float64).reshape(-1, 16, 16)
    lo = START_FRAC * numpy.maximum(d + g, 1e-3) - g
    return numpy.maximum(d + sd[:, None, None] * y, lo)


def loss_and_grad(params, x, target):
    """MSE over all outputs and its gradient as a packed vector."""
    ws = unpack(params)
    acts = forward(params, x)
    y = acts[3]
    n = y.size
    loss = float(numpy.mean((y - target) ** 2))
    g = 2.0 * (y - target) / n
    grads = [None] * 4
    for li in range(3, -1, -1):
        inp = acts[li - 1] if li > 0 else x
        grads[li] = conv_wgrad(inp, g)
        if li == 0:
            break
        g = conv_xgrad(g, ws[li][0]) * (inp > 0.0)
    return loss, pack(grads)


def adam(w, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One bias-corrected Adam step; returns new (w, m, v)."""
    m = b1 * m + (1.0 - b1) * g
    v = b2 * v + (1.0 - b2) * g * g
    w = w - lr * (m / (1.0 - b1 ** step)) / (numpy.sqrt(v / (1.0 - b2 ** step)) + eps)
    return w, m, v
