"""CPU checks of the normalised single-pixel variant's oracle
(oracle/normalized_ref.py) and host helpers.

The reference package is MATLAB and cannot run here, so the oracle is pinned
by construction instead: its segmentation against a literal port of
segpadimg.m / segimg.m, its noise term (FFT form, calcost.m) against the
matrix form u'Qu / sum(u) the kernel uses, its gradient and Hessian against
central finite differences, and the product's odd-size genfilter against the
oracle's.
"""
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
