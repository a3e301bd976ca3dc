"""CPU checks of the normalised single-pixel variant's oracle
(oracle/normalized_ref.py) and host helpers.

The reference package is MATLAB and cannot run here, so the oracle is pinned
by construction instead: its segmentation against a literal port of
segpadimg.m / segimg.m, its noise term (FFT form, calcost.m) against the
matrix form u'Qu / sum(u) the kernel uses, its gradient and Hessian against
central finite differences, and the product's odd-size genfilter against the
oracle's.
"""
import math

import numpy
import pytest

from oracle import normalized_ref as nr


def segpadimg_port(img, R1=1):
    """segpadimg.m + segimg.m ("matlab - single pixel with normalization/"),
    0-based: overlapping strips, replicate pad, R1+2 blocks stored transposed
    in column-major block order."""
    sz = img.shape[0]
    Ns = sz // R1
    ims0 = [img[:, 0:R1 + 1]]
    for ii in range(2, Ns):
        ims0.append(img[:, (ii - 1) * R1 - 1:ii * R1 + 1])
    ims0.append(img[:, (Ns - 1) * R1 - 1:Ns * R1])
    ims0 = numpy.concatenate(ims0, axis=1)
    ims1 = [ims0[0:R1 + 1, :]]
    for ii in range(2, Ns):
        ims1.append(ims0[(ii - 1) * R1 - 1:ii * R1 + 1, :])
    ims1.append(ims0[(Ns - 1) * R1 - 1:Ns * R1, :])
    ims2 = numpy.pad(numpy.concatenate(ims1, axis=0), 1, "edge")
    R = R1 + 2
    out = []
    for ii in range(Ns):                       # column strip
        tmp = ims2[:, ii * R:(ii + 1) * R]
        for k in range(Ns):                    # blocks of tmp' in column-major order
            out.append(tmp[k * R:(k + 1) * R, :].T)
    return out


def test_segments_match_segpadimg():
    rng = numpy.random.default_rng(0)
    img = rng.uniform(0, 50, size=(7, 7))
    ours = nr.segments(img)
    theirs = segpadimg_port(img)
    for ii in range(7):
        for k in range(7):
            # segment (strip ii, block k) belongs to pixel (k, ii), stored transposed
            assert numpy.array_equal(theirs[ii * 7 + k].T, ours[k * 7 + ii].reshape(3, 3))


def random_segment(seed):
    rng = numpy.random.default_rng(seed)
    d = rng.uniform(5, 80, size=(3, 3))
    g = rng.exponential(10, size=(3, 3)) + 0.5
    u = d + rng.normal(0, 2, size=(3, 3))
    return d, g, u


def test_matrix_form_of_the_noise_term():
    mask = nr.default_mask(0.1, 1.4, 0.7)
    Q = nr.q_matrix(mask)
    for seed in range(5):
        _, _, u = random_segment(seed)
        v = u.ravel()
        assert numpy.isclose(v @ Q @ v / v.sum(), nr.noise(u, mask), rtol=1e-12)
    assert numpy.allclose(Q, Q.T)


def test_gradient_and_hessian_vs_finite_differences():
    mask = nr.default_mask(0.1, 1.2, 0.6)
    Q = nr.q_matrix(mask)
    d, g, u = random_segment(7)
    alpha = 1.3
    f = lambda v: nr.cost(v.reshape(3, 3), d, g, mask, alpha)
    gr, Hm = nr.grad_hess(u.ravel(), d.ravel(), g.ravel(), Q, alpha)
    h = 1e-6
    for i in range(9):
        e = numpy.zeros(9)
        e[i] = h
        fd = (f(u.ravel() + e) - f(u.ravel() - e)) / (2 * h)
        assert abs(fd - gr[i]) <= 1e-6 * max(1.0, abs(gr[i]))
        gp, _ = nr.grad_hess(u.ravel() + e, d.ravel(), g.ravel(), Q, alpha)
        gm, _ = nr.grad_hess(u.ravel() - e, d.ravel(), g.ravel(), Q, alpha)
        assert numpy.allclose((gp - gm) / (2 * h), Hm[:, i], rtol=1e-5, atol=1e-8)


def test_newton_reaches_a_stationary_point():
    mask = nr.default_mask(0.1, 1.4, 0.7)
    Q = nr.q_matrix(mask)
    for seed in range(4):
        d, g, _ = random_segment(seed)
        u, fu = nr.newton(d, g, mask, 1.0)
        gr, _ = nr.grad_hess(u.ravel(), d.ravel(), g.ravel(), Q, 1.0)
        assert numpy.abs(gr).max() <= 1e-10
        assert fu <= nr.cost(d, d, g, mask, 1.0)


def test_product_mask_functions_match_the_oracle():
    from ncs_b200 import otf
    for t in (None, "pureN", "adjustable"):
        assert numpy.allclose(otf.genfilter_odd(3, 0.1, 2.8, 0.7, t),
                              nr.genfilter_odd(3, 0.1, 2.8, 0.7, t), rtol=0, atol=1e-15)
    assert numpy.allclose(otf.normalized_mask(0.1, 1.4, 0.7), nr.default_mask(0.1, 1.4, 0.7))
    m = otf.normalized_mask(0.1, 1.4, 0.7)
    assert m[1, 1] == 0.0 and numpy.allclose(m, m.T) and numpy.allclose(m, m[::-1, ::-1])


# A known answer derived by hand from calcost.m:36-53 for one 3 x 3 segment.
# u = d = [[2, 3, 1], [1, 1, 1], [1, 1, 1]], gamma = var / gain^2 = 2 / 1,
# alpha = 1/2, centred mask M = [[1, 2, 1], [1, 1/2, 1], [1, 2, 1]].
#   likelihood = sum(u - (d + gamma) log(u + gamma))
#              = (2 - 4 ln 4) + (3 - 5 ln 5) + 7 (1 - 3 ln 3)
#   fft2(u): u - 1 has 1 at (0, 0) and 2 at (0, 1), so
#   F(k1, k2) = 9 [k = 0] + 1 + 2 exp(-2 pi i k2 / 3):  |F(0, 0)| = 12,
#   |F(k1, 0)| = 3 for k1 = 1, 2, and |F(k1, k2)| = sqrt(3) for k2 = 1, 2.
#   fftshift moves frequency k to centred index (k + 1) mod 3 on each axis,
#   so |F| / 3 is 4 at M[1][1] = 1/2, 1 at M[0][1] = M[2][1] = 2, and
#   1 / sqrt(3) at the six entries of columns 0 and 2 (all 1):
#   sum((|F| / 3 M)^2) = 16 / 4 + 2 * 4 + 6 / 3 = 14, sum(u) = 12,
#   noisepart = 14 / 12 = 7 / 6;
#   fcost = 2 likelihood / 9 + alpha 7 / 6.
KNOWN_U = [[2.0, 3.0, 1.0], [1.0, 1.0, 1.0], [1.0, 1.0, 1.0]]
KNOWN_MASK = [[1.0, 2.0, 1.0], [1.0, 0.5, 1.0], [1.0, 2.0, 1.0]]
KNOWN_COST = (2.0 / 9.0) * (12.0 - 4.0 * math.log(4.0) - 5.0 * math.log(5.0)
                            - 21.0 * math.log(3.0)) + 0.5 * 7.0 / 6.0


def test_cost_known_answer_from_calcost():
    """The oracle's cost equals the value derived by hand above, line by line
    from calcost.m; a transposed mask (the wrong fftshift orientation) gives
    a different value, so the orientation is pinned too."""
    from oracle import normalized_ref as nr
    u = numpy.array(KNOWN_U)
    mask = numpy.array(KNOWN_MASK)
    assert abs(nr.noise(u, mask) - 7.0 / 6.0) <= 1e-14
    assert abs(nr.cost(u, u, 2.0, mask, 0.5) - KNOWN_COST) <= 1e-13 * abs(KNOWN_COST)
    assert abs(nr.noise(u, mask.T) - 7.0 / 6.0) > 0.1
