"""GPU tests of the simulator kernels (ncsb_sim_render, ncsb_sim_camera,
ncsb_sim_uniforms).

* rendering equals the host renderer (ncs_b200/sim.py render, FP64) to FP32
  rounding;
* the generator's uniforms, the Poisson sampler (inversion below 10, PTRS
  above) and the Gaussian read noise follow their distributions: moments
  within 6 standard errors and chi-square / Kolmogorov-Smirnov tests against
  the exact distributions at p > 1e-6, for fixed seeds;
* draws are a function of (seed, frame, pixel) only;
* the raw-ADU output solved through the preprocessing prologue equals the
  photo-electron output solved directly.
"""
import numpy
import pytest
import torch
from scipy import stats

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sim(cuda_ok):
    from ncs_b200 import sim
    return sim


def test_render_matches_host_renderer(sim):
    rng = numpy.random.default_rng(3)
    H, W = 93, 130
    chains = sim.wlc_emitters(3, 13.0, rng) / 0.1
    beads = rng.uniform(-8, 140, size=(60, 2))
    em = numpy.concatenate([chains, beads])
    photons = rng.uniform(50, 2000, size=len(em))
    ref = sim.render(em, H, W, 1.05, photons, 7.5).astype(numpy.float32)
    got = sim.render_gpu(em, H, W, 1.05, photons, 7.5).cpu().numpy()
    assert numpy.abs(got - ref).max() <= 1e-6 * numpy.abs(ref).max()


def lib():
    from ncs_b200 import _lib
    return _lib.load()


def uniforms(n, frame, seed):
    import ctypes
    out = torch.empty(n, dtype=torch.float32, device="cuda")
    assert lib().ncsb_sim_uniforms(n, frame, seed, ctypes.c_void_p(out.data_ptr()),
                                   ctypes.c_void_p(0)) == 0
    torch.cuda.synchronize()
    return out.cpu().numpy().astype(numpy.float64)


def test_uniforms(sim):
    u = uniforms(1 << 22, 0, 12345)
    n = u.size
    assert 0.0 < u.min() and u.max() < 1.0
    assert abs(u.mean() - 0.5) <= 6 * numpy.sqrt(1 / 12 / n)
    counts = numpy.bincount((u * 256).astype(int), minlength=256)
    assert stats.chisquare(counts).pvalue > 1e-6
    # neighbouring counters and another frame are not correlated
    assert abs(numpy.corrcoef(u[:-1], u[1:])[0, 1]) <= 6 / numpy.sqrt(n)
    v = uniforms(1 << 22, 1, 12345)
    assert abs(numpy.corrcoef(u, v)[0, 1]) <= 6 / numpy.sqrt(n)
    assert numpy.array_equal(u, uniforms(1 << 22, 0, 12345))
    assert not numpy.array_equal(u, uniforms(1 << 22, 0, 12346))


def counts(sim, lam, n_side=1024, seed=7):
    """Poisson draws only: gain 1, offset 0, no read noise -> ADU = n."""
    ideal = torch.full((n_side, n_side), lam, dtype=torch.float32, device="cuda")
    z = numpy.zeros((n_side, n_side))
    _, adu = sim.camera_gpu(ideal, 1, z, numpy.ones_like(z), z, seed, adu=True, photons=False)
    a = adu.cpu().numpy().ravel()
    assert numpy.array_equal(a, numpy.round(a))
    return a.astype(numpy.int64)


@pytest.mark.parametrize("lam", [0.3, 2.0, 9.99, 10.0, 37.5, 400.0])
def test_poisson_sampler(sim, lam):
    k = counts(sim, lam)
    n = k.size
    assert abs(k.mean() - lam) <= 6 * numpy.sqrt(lam / n)
    assert abs(k.var() - lam) <= 6 * numpy.sqrt((lam + 2 * lam * lam) / n)
    # chi-square against the exact pmf over the bins with >= 20 expected
    kmax = int(lam + 12 * numpy.sqrt(lam) + 20)
    obs = numpy.bincount(numpy.minimum(k, kmax), minlength=kmax + 1).astype(float)
    exp = n * stats.poisson.pmf(numpy.arange(kmax + 1), lam)
    exp[-1] += n * stats.poisson.sf(kmax, lam)
    ok = exp >= 20
    o = numpy.append(obs[ok], obs[~ok].sum())
    e = numpy.append(exp[ok], exp[~ok].sum())
    if e[-1] < 20:
        o[-2] += o[-1]
        e[-2] += e[-1]
        o, e = o[:-1], e[:-1]
    chi2 = ((o - e) ** 2 / e).sum()
    assert stats.chi2.sf(chi2, len(o) - 1) > 1e-6, (lam, chi2, len(o))


def test_read_noise_is_gaussian(sim):
    n_side = 1024
    ideal = torch.zeros((n_side, n_side), dtype=torch.float32, device="cuda")
    z = numpy.zeros((n_side, n_side))
    _, adu = sim.camera_gpu(ideal, 1, z + 3.0, numpy.ones_like(z), z + 4.0, 99, adu=True,
                            photons=False)
    x = (adu.cpu().numpy().ravel().astype(numpy.float64) - 3.0) / 2.0
    n = x.size
    assert abs(x.mean()) <= 6 / numpy.sqrt(n)
    assert abs(x.var() - 1.0) <= 6 * numpy.sqrt(2.0 / n)
    assert stats.kstest(x, "norm").pvalue > 1e-6


def test_camera_frames_and_photo_electrons(sim):
    w = sim.make_stack_gpu("frame256", T=64, seed=8, adu=True)
    phot, adu = w["images"], w["adu"]
    # frames are independent draws; the mean over frames approaches the ideal
    mean = adu.mean(0)
    expect = w["ideal"] * w["gain"] + w["offset"]
    sd = torch.sqrt(w["ideal"] * w["gain"] ** 2 + w["var"]) / 8.0
    assert ((mean - expect).abs() / sd).max().item() < 6.0
    # photo-electrons are the ADU conversion of the same draws
    d = (adu - w["offset"]) / w["gain"]
    d = torch.where(d <= 0, torch.full_like(d, 1e-6), d)
    assert torch.equal(d, phot)
    assert not torch.equal(adu[0], adu[1])


def test_simulated_raw_frames_through_the_fused_prologue(sim):
    import ncs_b200
    w = sim.make_stack_gpu("frame256", T=2, seed=9, adu=True)
    s = ncs_b200.Solver(alpha=w["alpha"])
    s.set_otf_mask(w["mask"])
    a = s.reduce_noise_adu(w["adu"], w["offset"], w["gain"], w["var"])
    g = (w["var"] / (w["gain"] * w["gain"])).contiguous()
    b = s.reduce_noise(w["images"], g)
    assert torch.equal(a, b)


def _sim_golden():
    import os
    return numpy.load(os.path.join(os.path.dirname(__file__), "golden", "sim_vectors.npz"))


def test_ideal_image_matches_the_reference_simulator(sim):
    """sim.ideal_image_gpu (device genpsfparam, occupancy, convolution,
    binning) against the reference's own genidealimage
    (python3-6/pyNCS/denoisetools.py:150-186) on its worm-like-chain
    positions (randwlcposition.mat): every pixel within 1e-6 of the image's
    maximum (FP32 kernel and output, FP64 sums)."""
    d = _sim_golden()
    for key in [k[:-len("_params")] for k in d.files if k.endswith("_params")]:
        R, zoom, px, na, lam = d[key + "_params"]
        got = sim.ideal_image_gpu(d["xcor"], d["ycor"], int(R), px, int(zoom), na, lam)
        ref = d[key + "_img"]
        err = numpy.abs(got.cpu().numpy().astype(numpy.float64) - ref).max()
        assert err <= 1e-6 * numpy.abs(ref).max(), (key, err)


def test_camera_moments_match_addnoise(sim):
    """The camera model against the reference's addnoise
    (python3-6/pyNCS/denoisetools.py:205-213) on the reference simulator's
    ideal image (I = 100 photons, bg = 10): E[ADU] = gain ideal + offset and
    Var[ADU] = gain^2 ideal + var per pixel (oracle/sim_ref.py), checked by
    the standardised residuals pooled over pixels and frames (mean within 6
    standard errors of 0, variance within 6 of 1), and per pixel the sample
    mean within 6 standard errors."""
    from oracle import sim_ref
    d = _sim_golden()
    ideal = d["R64_z4_img"] * 100.0 + 10.0
    R = ideal.shape[0]
    rng = numpy.random.default_rng(17)
    offset = rng.normal(100.0, 2.0, size=(R, R))
    gain = rng.normal(2.0, 0.2, size=(R, R))
    var = rng.exponential(60.0, size=(R, R))
    T = 400
    _, adu = sim.camera_gpu(torch.as_tensor(ideal, dtype=torch.float32, device="cuda"), T,
                            offset, gain, var, seed=99, adu=True, photons=False)
    a = adu.cpu().numpy().astype(numpy.float64)
    mean, variance = sim_ref.camera_moments(ideal.astype(numpy.float32).astype(numpy.float64),
                                            gain.astype(numpy.float32),
                                            var.astype(numpy.float32),
                                            offset.astype(numpy.float32))
    z = (a - mean) / numpy.sqrt(variance)
    n = z.size
    assert abs(z.mean()) <= 6 / numpy.sqrt(n)
    assert abs(z.var() - 1.0) <= 6 * numpy.sqrt(2.0 / n)
    per_pixel = (a.mean(axis=0) - mean) / numpy.sqrt(variance / T)
    assert numpy.abs(per_pixel).max() <= 6.0
