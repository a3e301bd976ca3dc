"""CPU tests: the oracle pinned against the reference's own outputs.

Golden vectors (tests/golden/reference_vectors.npz) were produced by
tests/golden/make_golden.py from the reference's Python (py_ref.py of
clib/pyCNCS/test and opencl/pyOpenCLNCS, ncs_c.py over the compiled
reference ncs.c, pyNCS genfilter).  Tolerances follow the reference tests:
clib/pyCNCS/test/test_sr.py (allclose; 1e-6 / 1e-5 on gradients; 1e-2 on
solutions) and test_im.py (allclose).
"""
import os

import numpy
import pytest

from conftest import create_otf_mask_shifted, random_otf_mask

GOLD = os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz")


@pytest.fixture(scope="module")
def gold():
    return numpy.load(GOLD)


def test_numpy_cost_terms_match_reference(gold):
    from oracle import numpy_ref as nr
    U, D, G = gold["cost_u"], gold["cost_data"], gold["cost_gamma"]
    ms = numpy.fft.fftshift(gold["cost_masks_centred"], axes=(-2, -1))
    a = float(gold["cost_alpha"])
    for i in range(U.shape[0]):
        assert numpy.allclose(nr.loglikelihood(U[i], D[i], G[i]), gold["cost_ll"][i],
                              rtol=1e-12)
        assert numpy.allclose(nr.noise(U[i], ms[i]), gold["cost_nc"][i], rtol=1e-12)
        assert numpy.allclose(nr.cost(U[i], D[i], G[i], ms[i], a), gold["cost_f"][i],
                              rtol=1e-12)


def test_gradients_match_reference_finite_differences(gold):
    """test_sr.py:55-97: LL gradient atol 1e-6, NC gradient atol 1e-5."""
    from oracle import numpy_ref as nr
    U, D, G = gold["cost_u"], gold["cost_data"], gold["cost_gamma"]
    ms = numpy.fft.fftshift(gold["cost_masks_centred"], axes=(-2, -1))
    for i in range(2):
        assert numpy.allclose(nr.ll_gradient(U[i], D[i], G[i]).ravel(), gold["fd_ll_grad"][i],
                              atol=1e-6 * 1e3)  # FD step 1e-6 on O(1e3) sums -> ~1e-3 noise
        assert numpy.allclose(nr.nc_gradient(U[i], ms[i]).ravel(), gold["fd_nc_grad"][i],
                              atol=1e-5 * 1e3)


def test_analytic_gradient_is_the_derivative():
    """Central differences in FP64 pin the analytic gradient tightly."""
    from oracle import numpy_ref as nr
    rng = numpy.random.default_rng(0)
    u = rng.uniform(1.0, 10.0, (16, 16))
    d = rng.uniform(1.0, 10.0, (16, 16))
    g = rng.uniform(2.0, 4.0, (16, 16))
    ms = create_otf_mask_shifted().astype(numpy.float64)
    grad = nr.gradient(u, d, g, ms, 0.3)
    h = 1e-5
    for (i, j) in [(0, 0), (3, 7), (15, 15), (8, 1)]:
        e = numpy.zeros_like(u)
        e[i, j] = h
        fd = (nr.cost(u + e, d, g, ms, 0.3) - nr.cost(u - e, d, g, ms, 0.3)) / (2 * h)
        assert abs(fd - grad[i, j]) < 1e-6


def test_c_oracle_cost_terms_match_reference(gold, oracle_libs):
    import ctypes
    lib = oracle_libs.load_port()
    U, D, G = gold["cost_u"], gold["cost_data"], gold["cost_gamma"]
    ms = numpy.fft.fftshift(gold["cost_masks_centred"], axes=(-2, -1))
    a = float(gold["cost_alpha"])
    for i in range(U.shape[0]):
        ll, nc = ctypes.c_double(), ctypes.c_double()
        f = lib.ncsp_cost(numpy.ascontiguousarray(U[i]), numpy.ascontiguousarray(D[i]),
                          numpy.ascontiguousarray(G[i]), numpy.ascontiguousarray(ms[i]), a, 16,
                          None, ctypes.byref(ll), ctypes.byref(nc))
        assert numpy.isclose(ll.value, gold["cost_ll"][i], rtol=1e-12)
        assert numpy.isclose(nc.value, gold["cost_nc"][i], rtol=1e-12)
        assert numpy.isclose(f, gold["cost_f"][i], rtol=1e-12)
    if oracle_libs.load_ref() is not None:
        sr = oracle_libs.NCSCSubRegion(16)
        for i in range(U.shape[0]):
            sr.newRegion(D[i], G[i])
            sr.setOTFMask(gold["cost_masks_centred"][i])
            sr.setU(U[i])
            assert numpy.isclose(sr.calcLogLikelihood(), gold["cost_ll"][i], rtol=1e-12)
            assert numpy.isclose(sr.calcNoiseContribution(), gold["cost_nc"][i], rtol=1e-12)
        sr.cleanup()


def test_solver_matches_scipy_reference(gold, oracle_libs):
    """test_sr.py:99-128: L-BFGS solution vs scipy L-BFGS-B, atol 1e-2."""
    for port in (True, False):
        for i in range(gold["solve_data"].shape[0]):
            ms = numpy.fft.fftshift(gold["solve_masks_centred"][i])
            u, ret, f = oracle_libs.solve_tile(gold["solve_data"][i], gold["solve_gamma"][i], ms,
                                               float(gold["solve_alpha"]), port=port)
            assert ret == 0
            assert numpy.allclose(u, gold["solve_u_scipy"][i], atol=1e-2)


def test_port_equals_reference_build(oracle_libs):
    if oracle_libs.load_ref() is None:
        pytest.skip("reference ncs.c not built here")
    rng = numpy.random.default_rng(4)
    img = rng.uniform(0.5, 80.0, (37, 29))
    gam = rng.uniform(1.0, 20.0, (37, 29))
    ms = create_otf_mask_shifted().astype(numpy.float64)
    a = oracle_libs.cReduceNoise(img, gam, ms, 0.1)
    b = oracle_libs.cReduceNoise(img, gam, ms, 0.1, port=True)
    assert numpy.array_equal(a, b)


def test_whole_image_tiling_matches_reference(gold, oracle_libs):
    """test_im.py:12-38: cReduceNoise and pyReduceNoise agree; our C oracle
    reproduces the reference wrapper's outputs (r_size 10, odd crops)."""
    if "im_c_0" not in gold:
        pytest.skip("golden image vectors absent")
    img, gam = gold["im_image"], gold["im_gamma"]
    om = gold["im_mask_centred"]
    for k, (ix, iy) in enumerate(gold["im_crops"]):
        assert numpy.allclose(gold["im_c_%d" % k], gold["im_py_%d" % k])
        got = oracle_libs.cReduceNoise(img[ix:, iy:], gam[ix:, iy:], numpy.fft.fftshift(om),
                                       float(gold["im_alpha"]), port=True)
        assert numpy.allclose(got, gold["im_c_%d" % k], rtol=1e-10, atol=1e-10)


def test_numpy_tiling_equals_c_loop():
    """tile_origins / segment / stitch restate ncs.c:66-143 exactly."""
    from oracle import numpy_ref as nr
    for n in range(14, 80):
        # the C loop of ncs.c:71-86 in padded coordinates
        want, i = [], -1
        while i < n + 1:
            b = n + 1 - 16 if i + 16 > n + 1 else i
            want.append(b + 1)
            if b == n + 1 - 16:
                break
            i += 14
        assert nr.tile_origins(n) == want
        # owner rule: the last covering tile
        o = nr.tile_origins(n)
        for y in range(n):
            owners = [b for b in o if b <= y < b + 14]
            assert owners and nr.owner_origin(y, o) == owners[-1]
    with pytest.raises(ValueError):
        nr.tile_origins(13)


def test_newton_optimum_is_stationary():
    from oracle import numpy_ref as nr
    rng = numpy.random.default_rng(9)
    d = rng.uniform(1.0, 200.0, (6, 16, 16))
    g = rng.exponential(15.0, (6, 16, 16)) + 0.5
    ms = create_otf_mask_shifted().astype(numpy.float64)
    u, f, its = nr.newton_solve(d, g, ms, 0.2)
    gr = nr.gradient(u, d, g, ms, 0.2)
    assert numpy.abs(gr).max() < 1e-7
    assert numpy.allclose(f, nr.cost(u, d, g, ms, 0.2), rtol=1e-12)
    # q_matrix is the quadratic form of the FFT noise term
    Q = nr.q_matrix(ms)
    x = rng.standard_normal((16, 16))
    assert numpy.isclose(x.ravel() @ Q @ x.ravel(), nr.noise(x, ms), rtol=1e-12)


def test_masks_match_reference(gold):
    from ncs_b200 import otf
    assert numpy.allclose(create_otf_mask_shifted(), gold["create_otf_mask_shifted"])
    numpy.random.seed(0)
    assert numpy.allclose(random_otf_mask(16, numpy.random), gold["random_mask_seed0"])
    for t in ("pureN", "adjustable", "OTFweighted"):
        assert numpy.allclose(otf.genfilter(16, 0.1, 1.4, 0.7, t), gold["genfilter_" + t])
    from ncs_b200.ncs import checkOTFMask
    m = otf.otf_weighted_mask()
    assert checkOTFMask(m)
    assert m[8, 8] == 0.0 and m.max() == 1.0


def test_genmaps_known_answer():
    """Three amplifiers, thresholds 100 and 200: pixels below 100 use pair 0,
    [100, 200) pair 1, >= 200 pair 2 (matlab/genmaps.m:36-58)."""
    from oracle import numpy_ref as nr
    adu = numpy.array([[[50.0, 100.0], [199.9, 200.0]]])
    gain = numpy.stack([numpy.full((2, 2), 1.0), numpy.full((2, 2), 2.0), numpy.full((2, 2), 4.0)])
    var = gain * 10.0
    g, v = nr.genmaps(adu, gain, var, (100.0, 200.0))
    assert numpy.array_equal(g[0], [[1.0, 2.0], [2.0, 4.0]])
    assert numpy.array_equal(v[0], [[10.0, 20.0], [20.0, 40.0]])
    off = numpy.full((2, 2), 100.0)
    d, gam = nr.adu_to_photons(adu, off, gain, var, (100.0, 200.0))
    # (50-100)/1 <= 0 -> 1e-6; (100-100)/2 = 0 -> 1e-6; 99.9/2; 100/4
    assert numpy.allclose(d[0], [[1e-6, 1e-6], [49.95, 25.0]])
    assert numpy.allclose(gam[0], [[10.0, 5.0], [5.0, 2.5]])
