"""FP64 restatement of the normalised single-pixel NCS variant (test
infrastructure: only the tests use it, as the checker of
ncsb_reduce_noise_normalized).

Reference: "matlab - single pixel with normalization/" in HuanglabPurdue/NCS
(MATLAB; it cannot run here, so this restatement is parity-unpinned against
the reference's own outputs -- it is checked against finite differences and
an independent matrix form of the same cost instead):
  * calcost.m:38-56     f(u) = 2 LL(u) / numel(u) + alpha * NC(u),
                        LL = sum(u - (d + gamma) log(u + gamma)),
                        NC = sum((|fftshift(fft2(u))| / n .* otfmask)^2) / sum(u),
                        gamma = var / gain^2;
  * reducenoise.m       Rs = 1: every pixel is its own 3 x 3 segment
                        (segpadimg.m: the pixel and its 8 neighbours,
                        replicate-padded at the frame border), minimised by
                        fminunc (quasi-Newton) from u = d for iterationN
                        iterations; stitchpadimg.m keeps each segment's centre;
                        out < 0 is set to 1e-6 (reducenoise.m, end of optimf);
  * genfilter.m:30-62   masks on the odd grid -(n-1)/2 .. (n-1)/2, default type
                        T = lambda / 2 / NA / 1.4, beta = 1, called with 2 NA
                        (reducenoise.m: otfsize = 2).
The referee here is an exact damped Newton solve (the cost is convex where
sum(u) > 0: a convex likelihood plus a quadratic-over-linear term).
"""
import numpy

N = 3  # segment side for Rs = 1


def genfilter_odd(n, pixelsize, NA, Lambda, type=None, w=1.0, h=0.7):
    """genfilter.m of the normalised variant (odd-size grid)."""
    r = numpy.arange(n) - (n - 1) / 2.0
    X, Y = numpy.meshgrid(r, r)
    scale = n * pixelsize
    kr = numpy.sqrt(X ** 2 + Y ** 2) / scale
    kmax = n / numpy.sqrt(2.0) / scale
    if type == "pureN":
        beta = 0.2
        T = (1 - beta) * Lambda / 2 / NA
    elif type == "adjustable":
        w0 = w * NA / Lambda
        beta = numpy.pi / 2 * (kmax / w0 - 1) / (numpy.arccos(1 - 2 * h) + numpy.pi / 2 * (kmax / w0 - 1))
        T = (1 - beta) / w0 / 2
    else:
        T = Lambda / 2 / NA / 1.4
        beta = 1.0
    rc = 0.5 * (1 + numpy.cos(numpy.pi * T / beta * (kr - (1 - beta) / 2 / T)))
    rc[kr < (1 - beta) / 2 / T] = 1
    rc[kr > (1 + beta) / 2 / T] = 0
    return 1 - rc


def default_mask(pixelsize, NA, Lambda):
    """The mask reducenoise.m builds with 10 arguments: genfilter(Rs+2, ...,
    otfsize*NA, Lambda), otfsize = 2."""
    return genfilter_odd(N, pixelsize, 2 * NA, Lambda)


def segments(img):
    """[H*W, 3, 3] segments of one frame in row-major pixel order: each pixel
    with its 8 neighbours, replicate padding (segpadimg.m with R1 = 1)."""
    img = numpy.asarray(img, dtype=numpy.float64)
    H, W = img.shape
    p = numpy.pad(img, 1, "edge")
    out = numpy.empty((H * W, N, N))
    for i in range(N):
        for j in range(N):
            out[:, i, j] = p[i:i + H, j:j + W].ravel()
    return out


def noise(u, mask_c):
    """NC(u) of calcost.m: sum((|fftshift(fft2(u))| / n * mask)^2) / sum(u)."""
    u = numpy.asarray(u, dtype=numpy.float64)
    F = numpy.abs(numpy.fft.fftshift(numpy.fft.fft2(u), axes=(-2, -1))) / N
    return ((F * mask_c) ** 2).sum(axis=(-2, -1)) / u.sum(axis=(-2, -1))


def cost(u, d, gamma, mask_c, alpha):
    u = numpy.asarray(u, dtype=numpy.float64)
    ll = (u - (d + gamma) * numpy.log(u + gamma)).sum(axis=(-2, -1))
    return 2.0 * ll / (N * N) + alpha * noise(u, mask_c)


def q_matrix(mask_c):
    """Q with sum((|fftshift(fft2(u))| / 3 * mask)^2) = u' Q u (u as a
    9-vector, row-major)."""
    mu = numpy.fft.ifftshift(numpy.asarray(mask_c, dtype=numpy.float64)) ** 2
    mu = 0.5 * (mu + numpy.roll(mu[::-1, ::-1], 1, axis=(0, 1)))  # symmetric part
    Q = numpy.zeros((N * N, N * N))
    e = numpy.eye(N * N)
    for a in range(N * N):
        Fa = numpy.fft.fft2(e[a].reshape(N, N))
        for b in range(N * N):
            Fb = numpy.fft.fft2(e[b].reshape(N, N))
            Q[a, b] = numpy.real((numpy.conj(Fa) * Fb * mu).sum()) / (N * N)
    return Q


def grad_hess(u, d, gamma, Q, alpha):
    """Gradient and Hessian of the cost at u (9-vectors)."""
    c = d + gamma
    a = u + gamma
    S = u.sum()
    Qu = Q @ u
    P = u @ Qu
    one = numpy.ones_like(u)
    g = 2.0 / 9.0 * (1.0 - c / a) + alpha * (2.0 * Qu * S - P) / S ** 2
    Hs = (2.0 * Q / S - 2.0 * (numpy.outer(Qu, one) + numpy.outer(one, Qu)) / S ** 2
          + 2.0 * P * numpy.outer(one, one) / S ** 3)
    Hm = 2.0 / 9.0 * numpy.diag(c / a ** 2) + alpha * Hs
    return g, Hm


def newton(d, gamma, mask_c, alpha, u0=None, iters=100, tol=1e-14):
    """Exact optimum of one segment (d, gamma: 3 x 3) by damped Newton with a
    feasibility-keeping backtracking line search."""
    Q = q_matrix(mask_c)
    d = numpy.asarray(d, dtype=numpy.float64).ravel()
    gamma = numpy.asarray(gamma, dtype=numpy.float64).ravel()
    u = d.copy() if u0 is None else numpy.asarray(u0, dtype=numpy.float64).ravel().copy()
    f = lambda v: cost(v.reshape(N, N), d.reshape(N, N), gamma.reshape(N, N), mask_c, alpha)
    fu = f(u)
    for _ in range(iters):
        g, Hm = grad_hess(u, d, gamma, Q, alpha)
        step = -numpy.linalg.solve(Hm, g)
        if numpy.abs(g).max() <= tol * max(1.0, numpy.abs(u).max()):
            break
        t = 1.0
        while t > 1e-12:
            un = u + t * step
            if (un + gamma > 0).all() and un.sum() > 0:
                fn = f(un)
                if fn <= fu + 1e-4 * t * (g @ step):
                    break
            t *= 0.5
        if t <= 1e-12:
            break
        u, fu = un, fn
    return u.reshape(N, N), fu


def reduce_noise(image, gamma, mask_c, alpha):
    """The variant's result for one frame at the exact per-segment optimum:
    each pixel's value is its segment's centre, values < 0 set to 1e-6.
    Returns (out [H, W], per-pixel optimal cost [H*W])."""
    image = numpy.asarray(image, dtype=numpy.float64)
    H, W = image.shape
    ds, gs = segments(image), segments(gamma)
    out = numpy.empty(H * W)
    fs = numpy.empty(H * W)
    for k in range(H * W):
        u, fs[k] = newton(ds[k], gs[k], mask_c, alpha)
        out[k] = u[1, 1]
    out[out < 0] = 1e-6
    return out.reshape(H, W), fs
