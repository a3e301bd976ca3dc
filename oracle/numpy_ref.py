"""FP64 numpy restatements of the NCS hot path -- TEST INFRASTRUCTURE ONLY.

Each function cites the reference code it restates (paths relative to the
HuanglabPurdue/NCS tree).  Everything here is float64 and batched over tiles
(leading axis).  Masks are *shifted* (DC at [0, 0]) unless a name says
``centred``.

  tile_origins / segment / stitch / owner_origin  <- ncs.c:66-143,
      ncs_c.py:296-319, cuda/pyCUDANCS/ncs.py:73-106, :161-171
  loglikelihood / ll_gradient                     <- ncs.c:158-208
  noise / nc_gradient                             <- ncs.c:220-299
  cost / gradient                                 <- ncs.c:335-364
  q_matrix                                        <- the quadratic form behind
      ncs.c:259-299: NC(u) = u^T Q u, Q = (1/N^2) F^H diag(M^2) F
  newton_solve                                    <- not in the reference: the
      exact FP64 optimum each tile's strictly convex cost has, used as referee.
"""
import numpy

FITMIN = 1.0e-6


# ---------------------------------------------------------------- tiling ---

def tile_origins(n, r=16):
    """Tile origins along one axis of length n, in padded (+1 halo) coordinates.

    ncs.c:71-86 walks i = -1, -1+(r-2), ... (unpadded) and shifts the last tile
    back so it ends at the padded edge; ncs.c:136-142 stops after that tile.
    """
    p = n + 2
    if p < r:
        raise ValueError("axis of length %d is smaller than the tile interior" % n)
    out = []
    b = 0
    while True:
        o = min(b, p - r)
        out.append(o)
        if o == p - r:
            break
        b += r - 2
    return out


def owner_origin(y, origins, r=16):
    """Origin of the tile whose interior value lands at frame index y: the last
    tile in row-major order whose interior [o, o + r - 2) covers y
    (ncs.c:121-130 overwrites in loop order)."""
    best = None
    for o in origins:
        if o <= y < o + r - 2:
            best = o
    return best


def segment(images, gamma, r=16):
    """Cut a [T,H,W] stack (gamma [H,W] shared, or [T,H,W]) into tiles.

    Returns (data [N,r,r], gamma [N,r,r], meta [N,3] = (frame, ox, oy)), tiles
    in (frame, ox, oy) row-major order, edge-replicated halo (numpy.pad 'edge'
    as ncs_c.py:297-298; ncs.c:88-113 clamps indices, which is the same)."""
    images = numpy.asarray(images, dtype=numpy.float64)
    if images.ndim == 2:
        images = images[None]
    gamma = numpy.asarray(gamma, dtype=numpy.float64)
    T, H, W = images.shape
    ox, oy = tile_origins(H, r), tile_origins(W, r)
    gpad = None if gamma.ndim == 3 else numpy.pad(gamma, 1, "edge")
    data, gam, meta = [], [], []
    for f in range(T):
        pim = numpy.pad(images[f], 1, "edge")
        pg = numpy.pad(gamma[f], 1, "edge") if gpad is None else gpad
        for a in ox:
            for b in oy:
                data.append(pim[a:a + r, b:b + r])
                gam.append(pg[a:a + r, b:b + r])
                meta.append((f, a, b))
    return numpy.array(data), numpy.array(gam), numpy.array(meta, dtype=numpy.int64)


def stitch(tiles, meta, shape, r=16):
    """Write each tile's interior to frame rows/cols [o, o + r - 2) in tile
    order, later tiles overwriting (ncs.c:121-130; ncs.py:161-171)."""
    T, H, W = shape
    out = numpy.zeros(shape, dtype=numpy.float64)
    for t, (f, a, b) in zip(tiles, meta):
        out[f, a:a + r - 2, b:b + r - 2] = t[1:-1, 1:-1]
    return out


# ------------------------------------------------------------- objective ---

def loglikelihood(u, data, gamma):
    """sum u - (d+g) log(max(u+g, 1e-6)) per tile (ncs.c:185-208)."""
    a = numpy.maximum(u + gamma, FITMIN)
    return numpy.sum(u - (data + gamma) * numpy.log(a), axis=(-2, -1))


def ll_gradient(u, data, gamma):
    """1 - (d+g)/max(u+g, 1e-6) (ncs.c:158-175)."""
    return 1.0 - (data + gamma) / numpy.maximum(u + gamma, FITMIN)


def noise(u, mask_shifted):
    """(1/N^2) sum |FFT2(u)|^2 M^2 (ncs.c:259-299)."""
    n2 = u.shape[-1] * u.shape[-2]
    uh = numpy.fft.fft2(u)
    return numpy.sum((uh.real ** 2 + uh.imag ** 2) * mask_shifted ** 2, axis=(-2, -1)) / n2


def nc_gradient(u, mask_shifted):
    """2 Q u = (1/N^2) IDFT(2 M^2 U) * N^2 / N^2 -- ncs.c:220-250 (c2r is
    unnormalised, then x 1/N^2)."""
    return numpy.real(numpy.fft.ifft2(2.0 * mask_shifted ** 2 * numpy.fft.fft2(u)))


def cost(u, data, gamma, mask_shifted, alpha):
    """f = LL + alpha NC (ncs.c:335-364)."""
    return loglikelihood(u, data, gamma) + alpha * noise(u, mask_shifted)


def gradient(u, data, gamma, mask_shifted, alpha):
    return ll_gradient(u, data, gamma) + alpha * nc_gradient(u, mask_shifted)


def q_kernel(mask_shifted):
    """q = ifft2(M^2): Q u = q (*) u, a 2-D circular convolution."""
    return numpy.real(numpy.fft.ifft2(mask_shifted ** 2))


def q_matrix(mask_shifted):
    """Dense Q with NC(u) = u^T Q u for u flattened row-major.

    Q[(x1,y1),(x2,y2)] = q[(x1-x2) mod r, (y1-y2) mod r]."""
    r = mask_shifted.shape[0]
    q = q_kernel(mask_shifted)
    x = numpy.arange(r)
    dx = (x[:, None] - x[None, :]) % r
    Q = q[dx[:, None, :, None], dx[None, :, None, :]]
    return Q.reshape(r * r, r * r)


# ---------------------------------------------------------- FP64 optimum ---

def newton_solve(data, gamma, mask_shifted, alpha, u0=None, max_iter=60, tol=1e-17):
    """Exact minimiser of each tile's cost by damped Newton in FP64.

    H = diag((d+g)/(u+g)^2) + 2 alpha Q is positive definite while u+g > 0
    and d+g > 0, so the optimum is unique.  Steps are limited to keep
    u+g >= 1e-3 (u+g) (strictly inside the log barrier) and backtracked on the
    exact cost.  Stops when the Newton decrement lambda^2/2 falls below
    tol * max(|f|, 1).  Returns (u*, f*, newton_iterations)."""
    data = numpy.asarray(data, dtype=numpy.float64)
    gamma = numpy.asarray(gamma, dtype=numpy.float64)
    squeeze = data.ndim == 2
    if squeeze:
        data, gamma = data[None], gamma[None]
    B, r, _ = data.shape
    n = r * r
    Q = q_matrix(mask_shifted)
    c = (data + gamma).reshape(B, n)
    g_ = gamma.reshape(B, n)
    u = (data if u0 is None else numpy.asarray(u0, dtype=numpy.float64)).reshape(B, n).copy()
    u = numpy.maximum(u, -g_ + 1e-3 * numpy.maximum(c, 1e-3))

    def fval(v, sel):
        a = numpy.maximum(v + g_[sel], FITMIN)
        return (numpy.sum(v - c[sel] * numpy.log(a), axis=1)
                + alpha * numpy.einsum("bi,ij,bj->b", v, Q, v))

    f = fval(u, slice(None))
    active = numpy.ones(B, dtype=bool)
    its = numpy.zeros(B, dtype=numpy.int64)
    for _ in range(max_iter):
        idx = numpy.nonzero(active)[0]
        if idx.size == 0:
            break
        ua = u[idx]
        a = ua + g_[idx]
        gr = 1.0 - c[idx] / a + 2.0 * alpha * ua @ Q
        H = 2.0 * alpha * numpy.broadcast_to(Q, (idx.size, n, n)).copy()
        H[:, numpy.arange(n), numpy.arange(n)] += c[idx] / a ** 2
        p = -numpy.linalg.solve(H, gr[..., None])[..., 0]
        lam2 = -numpy.sum(gr * p, axis=1)
        done = lam2 * 0.5 <= tol * numpy.maximum(numpy.abs(f[idx]), 1.0)
        # feasibility-limited, backtracked step
        neg = p < 0
        lim = numpy.where(neg, -(a * 0.999) / numpy.where(neg, p, -1.0), numpy.inf)
        t = numpy.minimum(1.0, lim.min(axis=1))
        fnew = numpy.empty(idx.size)
        for _k in range(60):
            trial = ua + t[:, None] * p
            fnew = fval(trial, idx)
            ok = fnew <= f[idx] - 0.25 * t * lam2 + 1e-12 * numpy.abs(f[idx])
            if ok.all():
                break
            t = numpy.where(ok, t, t * 0.5)
        take = ~done
        u[idx[take]] = (ua + t[:, None] * p)[take]
        f[idx[take]] = fnew[take]
        its[idx[take]] += 1
        active[idx[done]] = False
    u = u.reshape(B, r, r)
    if squeeze:
        return u[0], f[0], its[0]
    return u, f, its


def rel_cost_gap(f, fstar):
    """|f - f*| / max(|f*|, 1): the per-tile accuracy measure (tile costs can be
    negative, so the denominator is floored at 1)."""
    return numpy.abs(numpy.asarray(f) - numpy.asarray(fstar)) / numpy.maximum(numpy.abs(fstar), 1.0)


def genmaps(adu, gain, var, levels):
    """Per-frame gain and variance maps of a multi-amplifier camera: each pixel
    takes pair 0 below levels[0], pair k for levels[k-1] <= ADU < levels[k], the
    last pair above the last threshold (matlab/genmaps.m:29-62; with one pair
    the maps are used as they are).  adu [T,H,W]; gain, var [L,H,W]."""
    adu = numpy.asarray(adu, dtype=numpy.float64)
    gain = numpy.asarray(gain, dtype=numpy.float64)
    var = numpy.asarray(var, dtype=numpy.float64)
    if gain.ndim == 2:
        gain, var = gain[None], var[None]
    lv = numpy.zeros(adu.shape, dtype=numpy.int64)
    for t in levels:
        lv += (adu >= t)
    H, W = adu.shape[1:]
    rows = numpy.arange(H)[:, None]
    cols = numpy.arange(W)[None, :]
    return gain[lv, rows, cols], var[lv, rows, cols]


def adu_to_photons(adu, offset, gain, var, levels=()):
    """(d, gamma) from raw frames: d = (ADU - offset) / gain with d <= 0 set to
    1e-6 (python3-6/pyNCS/denoisetools.py:222-224), gamma = var / gain^2
    (denoisetools.py:266), the maps picked per pixel by genmaps."""
    g, v = genmaps(adu, gain, var, levels)
    d = (numpy.asarray(adu, dtype=numpy.float64) - numpy.asarray(offset, dtype=numpy.float64)) / g
    d[d <= 0] = 1e-6
    return d, v / (g * g)
