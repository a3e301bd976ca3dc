"""CPU tests of the GPU algorithm's numpy mirror (oracle/gpu_mirror.py).

The mirror restates the plain kernel's algorithm.  On a synthetic 512x512
frame (worm-like chains, sCMOS camera model, 2 % of pixels clamped to 1e-6)
with the workload's cap of 20 iterations, every tile must end within 1e-4
relative cost of the FP64 optimum.  Tiles with a clamped dark pixel and tiny
gamma are the hard case: without the fraction-to-barrier rule an Armijo-only
search steps into the FITMIN-clamped region and stalls (status -4)."""
import numpy


def test_mirror_reaches_optimum_on_synthetic_frame():
    from ncs_b200 import sim
    from oracle import gpu_mirror as gm
    from oracle import numpy_ref as nr
    w = sim.make_stack("stack512", T=1, device="cpu", seed=1234)
    td, tg, _ = nr.segment(w["images"].numpy(), w["gamma"].numpy())
    ms = numpy.fft.fftshift(w["mask"]).astype(numpy.float32).astype(numpy.float64)
    u, it, st, ev = gm.solve(td, tg, ms, 0.2, max_iters=20)
    assert set(numpy.unique(st)) <= {0, -2}
    sel = numpy.arange(0, td.shape[0], 3)
    _, fs, _ = nr.newton_solve(td[sel], tg[sel], ms, 0.2)
    gap = nr.rel_cost_gap(nr.cost(u[sel].astype(numpy.float64), td[sel], tg[sel], ms, 0.2), fs)
    assert gap.max() <= 1e-4
    # the hard tiles exist in this frame
    dark = (td <= 1e-6).any(axis=(1, 2)) & (tg < 0.05).any(axis=(1, 2))
    assert dark.any()


def test_mirror_barrier_rule_on_dark_pixel():
    """A single tile with a clamped dark pixel of tiny gamma next to bright
    pixels converges to the optimum."""
    from oracle import gpu_mirror as gm
    from oracle import numpy_ref as nr
    from ncs_b200 import otf
    rng = numpy.random.default_rng(2)
    d = rng.uniform(20.0, 60.0, (1, 16, 16))
    g = rng.uniform(5.0, 20.0, (1, 16, 16))
    d[0, 7, 7], g[0, 7, 7] = 1e-6, 0.01
    ms = numpy.fft.fftshift(otf.otf_weighted_mask())
    u, it, st, ev = gm.solve(d, g, ms, 0.2, max_iters=200, eps=1e-6)
    _, fs, _ = nr.newton_solve(d, g, ms, 0.2)
    assert st[0] == 0
    assert nr.rel_cost_gap(nr.cost(u.astype(numpy.float64), d, g, ms, 0.2), fs)[0] <= 1e-7
    assert (u + g).min() > 0


def test_mirror_stopping_rule_edge_cases():
    """The converged() cases of opencl/pyOpenCLNCS/test/test_solver_fns.py:63-110
    (||g|| / max(||x||, 1) against 1e-4): x = 0.9 with g = 1e-4 is not
    converged, x = 1.1 is, and x = 0.1/16 with g = 0.9e-4/16 is through the
    floor of 1 on ||x||.  With alpha 0 the gradient at a start x is
    1 - (d + gamma)/(x + gamma), so d is chosen to give that g; with no
    iterations allowed the status is the stopping test's verdict."""
    from conftest import create_otf_mask_shifted
    from oracle import gpu_mirror as gm
    for (x_val, g_val), expect in [((0.9, 1e-4), gm.MAXITERS), ((1.1, 1e-4), gm.SUCCESS),
                                   ((0.1 / 16, 0.9e-4 / 16), gm.SUCCESS)]:
        d = numpy.full((1, 16, 16), (1.0 - g_val) * (x_val + 1.0) - 1.0, numpy.float32)
        g = numpy.ones((1, 16, 16), numpy.float32)
        x = numpy.full((1, 16, 16), x_val, numpy.float32)
        _, it, st, _ = gm.solve(d, g, create_otf_mask_shifted(), 0.0, max_iters=0, eps=1e-4,
                                u0=x)
        assert st[0] == expect and it[0] == 0


