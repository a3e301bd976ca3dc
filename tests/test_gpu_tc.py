"""GPU tests of the tensor-core forms (NCSB_MODE_TC_TF32, NCSB_MODE_TC_BF16X3):
the spectral solve with every 16x16 transform of the noise term done as
tcgen05 GEMMs, TF32 operands or a three-way BF16 split, FP32 accumulation.

Each result is checked against the FP64 oracle, and each variant's error is
stated where it is measured:
* the noise term alone: at the start u = d, the kernel's cost f(d) = LL(d) +
  alpha d'Q d (its Q d from the GEMMs) against FP64, the error relative to
  the noise term alpha d'Q d within 8 units of the operands' rounding: TF32
  (10-bit mantissa) 8 x 2^-11 = 3.9e-3, BF16x3 8 x 2^-17 = 6.1e-5, the FP32
  FFT of the spectral form 64 x 2^-24 = 3.8e-6;
* whole solves: every tile's exact FP64 cost at the returned u within 1e-4
  relative of the FP64 Newton optimum (tiles of the reference's own test,
  the 2048-sensor workload's hot pixels); per pixel against the optimum and
  against pyCNCS: within 1e-3 for BF16x3, within 3e-2 for TF32 (its
  transform error moves the solution along directions in which the cost is
  flat: the cost gap stays below 1e-6);
* the stack path (device segmentation and stitching) equals the tile path.
Relative cost gap = |f - f*| / max(|f*|, 1).
"""
import numpy
import pytest
import torch

from conftest import create_otf_mask_shifted, random_otf_mask

pytestmark = pytest.mark.gpu

TC_FORMS = ["tc_tf32", "tc_bf16x3"]
# bound on |f_kernel(d) - f(d)| / (alpha d'Q d) for the start cost, per form
START_TOL = {"tc_tf32": 8 * 2.0 ** -11, "tc_bf16x3": 8 * 2.0 ** -17, "spectral": 64 * 2.0 ** -24}
# per-pixel agreement of converged solves (relative to max(|u|, 1))
PIXEL_TOL = {"tc_tf32": 3e-2, "tc_bf16x3": 1e-3}


@pytest.fixture(scope="module")
def ncs(cuda_ok):
    import ncs_b200
    return ncs_b200


def tiles_seed1(n):
    """data U(10,20), gamma U(2,4) -- cuda/pyCUDANCS/test/test_solver.py:79-84."""
    numpy.random.seed(1)
    data = numpy.random.uniform(10.0, 20.0, size=(n, 16, 16)).astype(numpy.float32)
    gamma = numpy.random.uniform(2.0, 4.0, size=(n, 16, 16)).astype(numpy.float32)
    return data, gamma


@pytest.mark.parametrize("form", TC_FORMS + ["spectral"])
def test_start_cost_measures_the_noise_term(ncs, form):
    """max_iters = 0: the solve stops after its first pass, which computes
    v = 2 alpha Q d with the GEMM stages (first-pass weights 2 alpha M^2),
    and reports f(d) = LL(d) + d'v / 2.  Random masks and a large alpha make
    the noise term a sizeable part of the cost."""
    from oracle import numpy_ref as nr
    rng = numpy.random.default_rng(3)
    n = 64
    data = rng.uniform(0.5, 400.0, size=(n, 16, 16)).astype(numpy.float32)
    gamma = rng.uniform(0.5, 40.0, size=(n, 16, 16)).astype(numpy.float32)
    worst = 0.0
    for trial in range(3):
        ms = numpy.fft.fftshift(random_otf_mask(16, rng)).astype(numpy.float32)
        alpha = [0.2, 1.0, 5.0][trial]
        s = ncs.Solver(alpha=alpha, max_iters=0, mode=form)
        s.set_otf_mask_shifted(ms)
        u, iters, status, cost = s.solve_tiles(torch.from_numpy(data).cuda(),
                                               torch.from_numpy(gamma).cuda())
        assert (status.cpu().numpy() == -2).all() and (iters.cpu().numpy() == 0).all()
        assert torch.equal(u.cpu(), torch.from_numpy(data))
        f64 = nr.cost(data.astype(numpy.float64), data.astype(numpy.float64),
                      gamma.astype(numpy.float64), ms.astype(numpy.float64), alpha)
        nc = alpha * nr.noise(data.astype(numpy.float64), ms.astype(numpy.float64))
        rel = numpy.abs(cost.cpu().numpy() - f64) / nc
        assert (nc / numpy.abs(f64)).min() > 1e-3  # the noise term matters here
        worst = max(worst, rel.max())
        s.close()
    assert worst <= START_TOL[form], worst
    print("%s: start cost max error %.2e of the noise term" % (form, worst))


@pytest.mark.parametrize("form", TC_FORMS)
def test_tiles_vs_fp64_optimum_and_spectral(ncs, oracle_libs, form):
    """Tiles of the reference's solver test, tight stopping rule: the exact
    FP64 cost at the returned u within 1e-6 relative of the optimum, pixels
    within 1e-3, the pyCNCS C solver's cost within 1e-4; iterations close to
    the spectral form's (the same algorithm, only the transforms differ)."""
    from oracle import numpy_ref as nr
    n, alpha = 64, 0.1
    data, gamma = tiles_seed1(n)
    ms = create_otf_mask_shifted()
    res = {}
    for f in (form, "spectral"):
        s = ncs.Solver(alpha=alpha, epsilon=1e-6, max_iters=500, mode=f)
        s.set_otf_mask_shifted(ms)
        u, it, st, cost = s.solve_tiles(torch.from_numpy(data).cuda(),
                                        torch.from_numpy(gamma).cuda())
        res[f] = (u.cpu().numpy().astype(numpy.float64), it.cpu().numpy(), st.cpu().numpy())
        s.close()
    u, it, st = res[form]
    assert (st == 0).all(), st
    ustar, fstar, _ = nr.newton_solve(data, gamma, ms.astype(numpy.float64), alpha)
    f_tc = nr.cost(u, data.astype(numpy.float64), gamma.astype(numpy.float64),
                   ms.astype(numpy.float64), alpha)
    gap = nr.rel_cost_gap(f_tc, fstar)
    assert gap.max() <= 1e-6, gap.max()
    pix = (numpy.abs(u - ustar) / numpy.maximum(numpy.abs(ustar), 1.0)).max()
    assert pix <= PIXEL_TOL[form], pix
    assert abs(it.mean() - res["spectral"][1].mean()) <= 1.0
    for i in range(0, n, 8):
        uref, ret, fref = oracle_libs.solve_tile(data[i].astype(numpy.float64),
                                                 gamma[i].astype(numpy.float64),
                                                 ms.astype(numpy.float64), alpha)
        assert nr.rel_cost_gap(f_tc[i], fref) <= 1e-4
    print("%s: max gap %.2e, max pixel error %.2e, mean iterations %.2f (spectral %.2f)"
          % (form, gap.max(), pix, it.mean(), res["spectral"][1].mean()))


@pytest.fixture(scope="module")
def sensor_crop(cuda_ok):
    from ncs_b200 import sim
    from oracle import numpy_ref as nr
    w = sim.make_stack("sensor2048", T=1, device="cuda", seed=2024, H=384, W=384, chains=4)
    td, tg, _ = nr.segment(w["images"].cpu().numpy(), w["gamma"].cpu().numpy())
    ms = numpy.fft.fftshift(w["mask"]).astype(numpy.float32).astype(numpy.float64)
    _, fstar, _ = nr.newton_solve(td, tg, ms, w["alpha"])
    return w, td, tg, ms, fstar


@pytest.mark.parametrize("form", TC_FORMS)
def test_sensor_crop_every_tile_and_stack_equals_tiles(ncs, sensor_crop, form):
    """The full-sensor workload's statistics (0.5 % hot pixels, variance x50)
    on 384 x 384, run to the stopping rule: all 784 tiles' exact costs within
    1e-4 of the FP64 optimum; the stack path (device segmentation and
    stitching) gives exactly the tile path's results."""
    from oracle import numpy_ref as nr
    w, td, tg, ms, fstar = sensor_crop
    s = ncs.Solver(alpha=w["alpha"], max_iters=w["max_iters"], mode=form)
    s.set_otf_mask(w["mask"])
    out, iters, status = s.reduce_noise(w["images"], w["gamma"], tile_stats="status")
    assert (status.cpu().numpy() == 0).all()
    u, it2, st2, _ = s.solve_tiles(torch.from_numpy(td.astype(numpy.float32)).cuda(),
                                   torch.from_numpy(tg.astype(numpy.float32)).cuda())
    assert torch.equal(it2, iters) and torch.equal(st2, status)
    ut = u.cpu().numpy().astype(numpy.float64)
    _, _, meta = nr.segment(w["images"].cpu().numpy(), w["gamma"].cpu().numpy())
    stitched = nr.stitch(ut, meta, tuple(w["images"].shape))
    assert numpy.array_equal(out.cpu().numpy().astype(numpy.float64), stitched)
    gap = nr.rel_cost_gap(nr.cost(ut, td, tg, ms, w["alpha"]), fstar)
    assert gap.size == 784 and gap.max() <= 1e-4, gap.max()
    print("%s sensor crop: max gap %.2e, mean iterations %.2f"
          % (form, gap.max(), iters.double().mean().item()))


@pytest.mark.parametrize("form", TC_FORMS)
def test_frame256_converged_vs_pycncs_pixels(ncs, oracle_libs, form):
    """1 frame 256 x 256, both run to ||g|| <= 1e-6 max(1, ||u||): the stitched
    frame within PIXEL_TOL relative per pixel of pyCNCS cReduceNoise
    (clib/pyCNCS/ncs_c.py:250-276)."""
    from ncs_b200 import sim
    w = sim.make_stack("frame256", device="cuda", seed=1234)
    img = w["images"][0].cpu().numpy().astype(numpy.float64)
    gam = w["gamma"].cpu().numpy().astype(numpy.float64)
    ms = numpy.fft.fftshift(w["mask"]).astype(numpy.float32).astype(numpy.float64)
    oracle_libs.set_overrides(epsilon=1e-6)
    try:
        ref = oracle_libs.cReduceNoise(img, gam, ms, w["alpha"])
    finally:
        oracle_libs.set_overrides()
    s = ncs.Solver(alpha=w["alpha"], epsilon=1e-6, max_iters=1000, mode=form)
    s.set_otf_mask(w["mask"])
    out, _, status = s.reduce_noise(w["images"], w["gamma"], tile_stats="status")
    assert (status.cpu().numpy() == 0).all()
    got = out[0].cpu().numpy().astype(numpy.float64)
    rel = numpy.abs(got - ref) / numpy.maximum(numpy.abs(ref), 1.0)
    assert rel.max() <= PIXEL_TOL[form], rel.max()
    print("%s frame256 vs pyCNCS: max pixel error %.2e" % (form, rel.max()))


@pytest.mark.parametrize("form", TC_FORMS)
def test_status_codes_nan_tile_and_odd_shapes(ncs, form):
    """A NaN pixel ends its own tile with a failure status and leaves the
    other tiles (including the ones sharing its CTA and its GEMM rows)
    unchanged; odd frame sizes and a tile count that is not a multiple of 8
    exercise the partly filled last CTA."""
    rng = numpy.random.default_rng(9)
    T, H, W = 3, 37, 53
    images = rng.uniform(1.0, 90.0, size=(T, H, W)).astype(numpy.float32)
    gamma = rng.uniform(0.5, 30.0, size=(H, W)).astype(numpy.float32)
    s = ncs.Solver(alpha=0.3, max_iters=100, mode=form)
    s.set_otf_mask_shifted(create_otf_mask_shifted())
    x = torch.from_numpy(images).cuda()
    g = torch.from_numpy(gamma).cuda()
    ref, rit, rst = s.reduce_noise(x, g, tile_stats="status")
    assert rit.numel() % 8 != 0
    assert (rst.cpu().numpy() == 0).all()
    bad = images.copy()
    bad[1, 20, 30] = numpy.nan
    out, it, st = s.reduce_noise(torch.from_numpy(bad).cuda(), g, tile_stats="status")
    st = st.cpu().numpy()
    failed = numpy.nonzero(st != 0)[0]
    assert 1 <= failed.size <= 4
    ok = numpy.ones(st.size, bool)
    ok[failed] = False
    assert (it.cpu().numpy()[ok] == rit.cpu().numpy()[ok]).all()
    # frames without the NaN pixel are unchanged
    assert torch.equal(out[0], ref[0]) and torch.equal(out[2], ref[2])
    # cap 0 and 1
    for cap in (0, 1):
        s.set_params(max_iters=cap)
        _, it, st = s.reduce_noise(x, g, tile_stats="status")
        assert (it.cpu().numpy() <= cap).all()
        assert set(numpy.unique(st.cpu().numpy())) <= {0, -2}


@pytest.mark.parametrize("form", TC_FORMS)
def test_warm_start_with_tc_form(ncs, form):
    """A proposed start through the tensor-core form: a tile whose proposal
    is worse than the photon image starts from the photon image, and its
    result equals the tensor-core solve without a proposal bit for bit."""
    rng = numpy.random.default_rng(21)
    T, H, W = 2, 40, 45
    images = rng.uniform(1.0, 90.0, size=(T, H, W)).astype(numpy.float32)
    gamma = rng.uniform(0.5, 30.0, size=(H, W)).astype(numpy.float32)
    s = ncs.Solver(alpha=0.2, max_iters=100, mode=form)
    s.set_otf_mask_shifted(create_otf_mask_shifted())
    x = torch.from_numpy(images).cuda()
    g = torch.from_numpy(gamma).cuda()
    ref, rit, rst = s.reduce_noise(x, g, tile_stats="status")
    n = rit.numel()
    from oracle import numpy_ref as nr
    td, _, _ = nr.segment(images, gamma)
    u0 = torch.from_numpy((td * 3.0 + 50.0).astype(numpy.float32)).cuda()  # bad proposals
    out, it, st, cost, ev, fb = s.reduce_noise_from(x, g, u0)
    assert (fb.cpu().numpy() == 1).all()
    assert torch.equal(out, ref) and torch.equal(it, rit)
    good = torch.from_numpy(td.astype(numpy.float32)).cuda()  # the photon image itself
    out2, it2, st2, _, _, fb2 = s.reduce_noise_from(x, g, good)
    assert (st2.cpu().numpy() == 0).all() and it2.numel() == n


@pytest.mark.parametrize("form", TC_FORMS)
def test_batch_equals_single_stack_solves(ncs, form):
    """The batched launch (many stacks, each with its own shape, alpha and
    mask, one queue) in a tensor-core form: every stack's result, iterations
    and status equal a single-stack solve of the same form bit for bit, with
    and without proposed starts; the batch can be captured in a CUDA graph."""
    from ncs_b200 import sim, warmstart
    stacks = sim.make_mixed(6, seed=31, sides=(64, 128), frames=(1, 3))
    ref = []
    for st in stacks:
        s1 = ncs.Solver(alpha=st["alpha"], max_iters=60, mode=form)
        s1.set_otf_mask(st["mask"])
        o, it, sta = s1.reduce_noise(st["images"], st["gamma"], tile_stats="status")
        ref.append((o, it, sta))
        s1.close()
    s = ncs.Solver(max_iters=60, mode=form)
    outs = s.batch_set(stacks)
    stats = s.batch_stats()
    s.batch_reduce_noise(stats=stats)
    torch.cuda.synchronize()
    off = 0
    for (o, it, sta), out in zip(ref, outs):
        n = it.numel()
        assert torch.equal(out, o)
        assert torch.equal(stats["iters"][off:off + n], it)
        assert torch.equal(stats["status"][off:off + n], sta)
        off += n
    assert off == s.batch_tiles
    # proposals from the batched network inference, solved in the same form
    net = warmstart.WarmStartNet.load()
    u0 = net.propose_batch(s)
    stats2 = s.batch_stats()
    s.batch_reduce_noise(u0_tiles=u0, stats=stats2)
    torch.cuda.synchronize()
    assert (stats2["status"].cpu().numpy() == 0).all()
    off = 0
    for st, out in zip(stacks, outs):
        s1 = ncs.Solver(alpha=st["alpha"], max_iters=60, mode=form)
        s1.set_otf_mask(st["mask"])
        n = s1.num_tiles(*st["images"].shape)
        o, it, sta, _, _, fb = s1.reduce_noise_from(st["images"], st["gamma"],
                                                    u0[off:off + n].contiguous())
        assert torch.equal(out, o) and torch.equal(stats2["iters"][off:off + n], it)
        assert torch.equal(stats2["start"][off:off + n], fb)
        off += n
        s1.close()
    # graph capture and replay of the batched launch
    graph = torch.cuda.CUDAGraph()
    stats3 = s.batch_stats()
    s.batch_reduce_noise(stats=stats3)  # warm-up outside the capture
    torch.cuda.synchronize()
    with torch.cuda.graph(graph):
        s.batch_reduce_noise(stats=stats3)
    for o in outs:
        o.zero_()
    graph.replay()
    torch.cuda.synchronize()
    for (o, it, sta), out in zip(ref, outs):
        assert torch.equal(out, o)
    del graph
    s.close()
