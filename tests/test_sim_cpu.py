"""CPU tests of the host simulator (ncs_b200/sim.py) against the physics the
synthetic workloads are specified with: worm-like chains with emitters every
20 nm and a 2 um persistence length, a pixel-integrated Gaussian PSF that
conserves each emitter's photons, and sCMOS maps with offset ~ N(100, 2) ADU,
gain ~ N(2.0, 0.2) and read variance ~ Exp(mean 60 ADU^2) (the camera model of
denoisetools.py:205-225 with per-pixel maps)."""
import math

import numpy


def test_wlc_chain_geometry():
    from ncs_b200 import sim
    rng = numpy.random.default_rng(0)
    em = sim.wlc_emitters(1, 50.0, rng, lp=2.0, length=(5.0, 5.0), spacing=0.02)
    steps = numpy.linalg.norm(numpy.diff(em, axis=0), axis=1)
    assert em.shape == (250, 2) and numpy.allclose(steps, 0.02)
    # tangent correlation: the turning angle per step ds has variance 2 ds / lp,
    # so over a contour length s, <cos dtheta> = exp(-s / lp); at s = 1 um
    # (50 steps) and lp = 2 um that is exp(-1/2), averaged here over 200 chains
    cs = []
    for k in range(200):
        e = sim.wlc_emitters(1, 50.0, numpy.random.default_rng(k), lp=2.0,
                             length=(5.0, 5.0), spacing=0.02)
        t = numpy.diff(e, axis=0)
        t /= numpy.linalg.norm(t, axis=1, keepdims=True)
        cs.append(numpy.mean(numpy.sum(t[:-50] * t[50:], axis=1)))
    assert abs(numpy.mean(cs) - math.exp(-0.5)) < 0.05


def test_psf_conserves_photons():
    from ncs_b200 import sim
    em = numpy.array([[20.3, 17.8], [30.0, 30.5]])
    img = sim.render(em, 48, 48, 1.05, 1000.0, 0.0)
    # a 11 x 11 window holds all but ~1e-6 of a sigma = 1.05 px Gaussian
    assert abs(img.sum() - 2000.0) < 0.01
    bg = sim.render(em, 48, 48, 1.05, 0.0, 7.5)
    assert numpy.allclose(bg, 7.5)
    # the centroid of one emitter's image sits at its position (pixel i spans [i, i+1))
    one = sim.render(em[:1], 48, 48, 1.05, 1000.0, 0.0)
    ys, xs = numpy.mgrid[0:48, 0:48] + 0.5
    assert abs((one * xs).sum() / one.sum() - 20.3) < 1e-3
    assert abs((one * ys).sum() / one.sum() - 17.8) < 1e-3


def test_camera_map_distributions():
    from ncs_b200 import sim
    off, gain, var = sim.camera_maps(512, 512, numpy.random.default_rng(1))
    assert abs(off.mean() - 100.0) < 0.02 and abs(off.std() - 2.0) < 0.02
    assert abs(gain.mean() - 2.0) < 0.002 and abs(gain.std() - 0.2) < 0.002
    assert abs(var.mean() - 60.0) < 0.5 and (var >= 0).all()
    # hot pixels: a fraction of the variance map scaled by 50
    _, _, vh = sim.camera_maps(512, 512, numpy.random.default_rng(1), hot=0.005)
    assert 0.003 < numpy.mean(vh > 1000.0) < 0.008


def test_ideal_image_restatement_matches_the_reference_simulator():
    """oracle/sim_ref.py's genidealimage restatement against the reference's
    own genidealimage outputs (tests/golden/sim_vectors.npz, written by
    make_sim_golden.py from denoisetools.py and randwlcposition.mat): grids
    of 32-128 pixels, zoom 1-8, three numerical apertures."""
    import os
    from oracle import sim_ref
    d = numpy.load(os.path.join(os.path.dirname(__file__), "golden", "sim_vectors.npz"))
    cases = [k[:-len("_params")] for k in d.files if k.endswith("_params")]
    assert len(cases) == 4
    for key in cases:
        R, zoom, px, na, lam = d[key + "_params"]
        img, k = sim_ref.ideal_image(d["xcor"], d["ycor"], int(R), px, int(zoom), na, lam)
        assert numpy.abs(k - d[key + "_kernel"]).max() <= 1e-15
        ref = d[key + "_img"]
        assert numpy.abs(img - ref).max() <= 1e-12 * numpy.abs(ref).max(), key
