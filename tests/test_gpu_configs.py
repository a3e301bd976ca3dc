"""GPU parity tests on the named workloads, each checked tile by tile against
the FP64 oracle:

* frame256 -- 1 frame 256 x 256, 12 worm-like chains, L-BFGS cap 15: every
  solver form at the cap against the FP64 Newton optimum (fraction of tiles
  converged, per-tile cost gap), beside the reference C path (pyCNCS
  ncs.c, ncsSRSolve per tile) at the same cap; and, run to a tight stopping
  rule, the whole frame against pyCNCS cReduceNoise
  (clib/pyCNCS/ncs_c.py:250-276) pixel by pixel.
* a 384 x 384 crop of the sensor workload -- 0.5 % hot pixels whose read
  variance is x50, run to the stopping rule: every tile of every form
  within 1e-4 relative cost of the FP64 optimum.
* a small mixed batch -- several ROI sides, alphas, numerical apertures and
  wavelengths in one batched launch: every tile within 1e-4 of the FP64
  optimum of its own stack's alpha and mask.

Relative cost gap = |f - f*| / max(|f*|, 1) (tile costs can be negative).
"""
import numpy
import pytest
import torch

pytestmark = pytest.mark.gpu

FORMS = ["spectral", "plain", "plain_wg"]


@pytest.fixture(scope="module")
def ncs(cuda_ok):
    import ncs_b200
    return ncs_b200


def _mask64(w):
    return numpy.fft.fftshift(w["mask"]).astype(numpy.float32).astype(numpy.float64)


@pytest.fixture(scope="module")
def frame256(cuda_ok):
    from ncs_b200 import sim
    from oracle import numpy_ref as nr
    w = sim.make_stack("frame256", device="cuda", seed=1234)
    td, tg, _ = nr.segment(w["images"].cpu().numpy(), w["gamma"].cpu().numpy())
    _, fstar, _ = nr.newton_solve(td, tg, _mask64(w), w["alpha"])
    return w, td, tg, fstar


@pytest.mark.parametrize("form", FORMS)
def test_frame256_at_the_cap_vs_fp64_and_pycncs(ncs, oracle_libs, frame256, form):
    """At the workload's cap of 15 iterations.  The spectral form converges
    every tile well inside the cap; the plain forms (the reference's scalar
    initial matrix) leave some tiles at the cap, and those still have to be
    within 1e-4 of the optimum.  The reference C path is run on every tile at
    the same cap: some of its capped tiles end above 1e-4 (1.6e-4 on this
    frame), and no form may end further from the optimum than it does."""
    from oracle import numpy_ref as nr
    w, td, tg, fstar = frame256
    cap = w["max_iters"]
    assert cap == 15 and td.shape[0] == 361
    s = ncs.Solver(alpha=w["alpha"], max_iters=cap, mode=form, m=1 if form == "spectral" else 4)
    s.set_otf_mask(w["mask"])
    out, iters, status, cost = s.reduce_noise(w["images"], w["gamma"], tile_stats=True)
    st = status.cpu().numpy()
    gap = nr.rel_cost_gap(cost.cpu().numpy(), fstar)
    converged = float((st == 0).mean())
    assert set(numpy.unique(st)) <= {0, -2}
    assert int(iters.max().item()) <= cap
    if form == "spectral":
        assert converged == 1.0
    assert gap.max() <= 1e-4, (converged, gap.max())

    # the reference C solver on every tile at the same cap
    ms = _mask64(w)
    oracle_libs.set_overrides(max_iterations=cap)
    try:
        ref = [oracle_libs.solve_tile(td[i], tg[i], ms, w["alpha"]) for i in range(len(td))]
    finally:
        oracle_libs.set_overrides()
    fref = numpy.array([r[2] for r in ref])
    ref_gap = nr.rel_cost_gap(fref, fstar)
    ref_converged = float(numpy.mean([r[1] == 0 for r in ref]))
    # at the same cap every form is at least as close to the optimum as the
    # reference C path (libLBFGS-API solver) on its worst tile, and converges
    # at least as many tiles
    assert gap.max() <= max(ref_gap.max(), 1e-6)
    if form == "spectral":
        assert converged >= ref_converged
    print("frame256 cap %d %s: converged %.3f, max gap %.2e | pyCNCS: converged %.3f, max gap "
          "%.2e" % (cap, form, converged, gap.max(), ref_converged, ref_gap.max()))


def test_frame256_converged_vs_pycncs_pixels(ncs, oracle_libs, frame256):
    """Both run to a tight stopping rule (||g|| <= 1e-6 max(1, ||u||)): the
    stitched frame agrees with pyCNCS cReduceNoise within 1e-3 relative per
    pixel (relative to max(|u|, 1))."""
    w, _, _, _ = frame256
    img = w["images"][0].cpu().numpy().astype(numpy.float64)
    gam = w["gamma"].cpu().numpy().astype(numpy.float64)
    oracle_libs.set_overrides(epsilon=1e-6)
    try:
        ref = oracle_libs.cReduceNoise(img, gam, _mask64(w), w["alpha"])
    finally:
        oracle_libs.set_overrides()
    for form in FORMS:
        s = ncs.Solver(alpha=w["alpha"], epsilon=1e-6, max_iters=1000, mode=form)
        s.set_otf_mask(w["mask"])
        out, _, status = s.reduce_noise(w["images"], w["gamma"], tile_stats="status")
        assert (status.cpu().numpy() == 0).all(), form
        got = out[0].cpu().numpy().astype(numpy.float64)
        rel = numpy.abs(got - ref) / numpy.maximum(numpy.abs(ref), 1.0)
        assert rel.max() <= 1e-3, (form, rel.max())


@pytest.fixture(scope="module")
def sensor_crop(cuda_ok):
    from ncs_b200 import sim
    from oracle import numpy_ref as nr
    w = sim.make_stack("sensor2048", T=1, device="cuda", seed=2024, H=384, W=384, chains=4)
    td, tg, _ = nr.segment(w["images"].cpu().numpy(), w["gamma"].cpu().numpy())
    _, fstar, _ = nr.newton_solve(td, tg, _mask64(w), w["alpha"])
    return w, fstar


@pytest.mark.parametrize("form", FORMS)
def test_sensor_crop_with_hot_pixels_every_tile(ncs, sensor_crop, form):
    """384 x 384 of the full-sensor workload: 0.5 % hot pixels (read variance
    x50), run to the stopping rule (200-iteration cap): all 784 tiles within
    1e-4 relative cost of the FP64 optimum."""
    from oracle import numpy_ref as nr
    w, fstar = sensor_crop
    gam = w["gamma"].cpu().numpy()
    assert (gam > 20 * numpy.median(gam)).mean() > 0.002  # the hot pixels are there
    s = ncs.Solver(alpha=w["alpha"], max_iters=w["max_iters"], mode=form,
                   m=1 if form == "spectral" else 4)
    s.set_otf_mask(w["mask"])
    out, iters, status, cost = s.reduce_noise(w["images"], w["gamma"], tile_stats=True)
    assert (status.cpu().numpy() == 0).all()
    gap = nr.rel_cost_gap(cost.cpu().numpy(), fstar)
    assert gap.size == 784 and gap.max() <= 1e-4, gap.max()


def test_mixed_batch_every_tile_vs_fp64(ncs):
    """A small mixed batch (ROI sides 64-256, 1-3 frames, each stack with its
    own alpha, NA, wavelength and so its own mask; chains or beads) in one
    batched launch: every tile within 1e-4 relative cost of the FP64 optimum
    for its own stack's alpha and mask."""
    from ncs_b200 import sim
    from oracle import numpy_ref as nr
    stacks = sim.make_mixed(8, seed=99, sides=(64, 128, 256), frames=(1, 3))
    assert len({st["alpha"] for st in stacks}) == 8
    assert len({(st["NA"], st["wavelength"]) for st in stacks}) > 1
    s = ncs.Solver(max_iters=200)
    s.batch_set(stacks)
    stats = s.batch_stats()
    s.batch_reduce_noise(stats=stats)
    torch.cuda.synchronize()
    cost = stats["cost"].cpu().numpy()
    assert (stats["status"].cpu().numpy() == 0).all()
    off = 0
    for st in stacks:
        td, tg, _ = nr.segment(st["images"].cpu().numpy(), st["gamma"].cpu().numpy())
        _, fstar, _ = nr.newton_solve(td, tg, _mask64(st), st["alpha"])
        gap = nr.rel_cost_gap(cost[off:off + len(td)], fstar)
        assert gap.max() <= 1e-4, (st["name"], gap.max())
        off += len(td)
    assert off == s.batch_tiles
