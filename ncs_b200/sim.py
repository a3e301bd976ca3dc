"""Seeded synthetic sCMOS stacks with the shapes and statistics of the named
NCS workloads (the reference's own simulation inputs -- calibration .mat
maps -- are not shipped, so these stand in for them).

Physics (all lengths in micrometres):
  * structure: worm-like chains, persistence length 2, contour length
    U(5, 10), tangent angle diffusing so that <cos> decays as exp(-s/Lp);
    emitters every 0.02 along each chain, ``photons`` each;
  * optics: Gaussian PSF sigma = 0.21 lambda / NA (lambda 0.7, NA 1.4 ->
    0.105 = 1.05 px at 0.1 px size), integrated over each pixel;
  * background ``bg`` photons / px, independent Poisson draw per frame;
  * camera (per pixel): offset ~ N(100, 2) ADU, gain ~ N(2, 0.2) ADU/e-,
    read variance ~ Exponential(mean 60 ADU^2); optional hot pixels whose
    variance is x50.  ADU = gain * photons + sqrt(var) N(0,1) + offset;
  * NCS inputs as python3-6/pyNCS/denoisetools.py:205-225: d = (ADU -
    offset) / gain with d <= 0 set to 1e-6, gamma = var / gain^2.
The ideal image and camera maps are drawn with numpy PCG64 (CPU, small);
frames are drawn with a seeded torch generator on the target device.
"""
import math

import numpy
import torch

from .otf import otf_weighted_mask

WORKLOADS = {
    # 1 frame 256x256, 12 chains, L-BFGS cap 15
    "frame256": dict(T=1, H=256, W=256, chains=12, photons=100.0, bg=10.0, hot=0.0,
                     alpha=0.2, max_iters=15),
    # 200 frames 512x512, shared gamma map, cap 20, all tiles in one launch
    "stack512": dict(T=200, H=512, W=512, chains=12, photons=100.0, bg=10.0, hot=0.0,
                     alpha=0.2, max_iters=20),
    # 100 frames 2048x2048, 60 chains, 0.5% hot pixels, run to the stopping rule
    "sensor2048": dict(T=100, H=2048, W=2048, chains=60, photons=100.0, bg=10.0, hot=0.005,
                       alpha=0.2, max_iters=200),
}


def wlc_emitters(n_chains, field, rng, lp=2.0, length=(5.0, 10.0), spacing=0.02):
    """Emitter positions (x, y) of n_chains 2-D worm-like chains in a square field."""
    out = []
    for _ in range(n_chains):
        L = rng.uniform(*length)
        n = max(int(L / spacing), 2)
        th0 = rng.uniform(0.0, 2.0 * math.pi)
        dth = rng.normal(0.0, math.sqrt(2.0 * spacing / lp), size=n)
        th = th0 + numpy.cumsum(dth)
        x = rng.uniform(0.0, field) + numpy.cumsum(spacing * numpy.cos(th))
        y = rng.uniform(0.0, field) + numpy.cumsum(spacing * numpy.sin(th))
        out.append(numpy.stack([x, y], axis=1))
    return numpy.concatenate(out, axis=0)


def render(emitters_px, H, W, sigma_px, photons, bg, half=5):
    """bg + photons * pixel-integrated Gaussian PSF at each emitter (px units,
    pixel i spans [i, i+1)); ``photons`` is a scalar or one value per emitter."""
    from scipy.special import erf
    img = numpy.full((H, W), float(bg))
    s2 = math.sqrt(2.0) * sigma_px
    ph = numpy.broadcast_to(numpy.asarray(photons, dtype=numpy.float64), (len(emitters_px),))
    for (x, y), photons in zip(emitters_px, ph):  # x along W (columns), y along H (rows)
        cx, cy = int(math.floor(x)), int(math.floor(y))
        cols = numpy.arange(cx - half, cx + half + 1)
        rows = numpy.arange(cy - half, cy + half + 1)
        px = 0.5 * (erf((cols + 1 - x) / s2) - erf((cols - x) / s2))
        py = 0.5 * (erf((rows + 1 - y) / s2) - erf((rows - y) / s2))
        rm = (rows >= 0) & (rows < H)
        cm = (cols >= 0) & (cols < W)
        if rm.any() and cm.any():
            img[numpy.ix_(rows[rm], cols[cm])] += photons * numpy.outer(py[rm], px[cm])
    return img


def camera_maps(H, W, rng, hot=0.0):
    offset = rng.normal(100.0, 2.0, size=(H, W))
    gain = rng.normal(2.0, 0.2, size=(H, W))
    var = rng.exponential(60.0, size=(H, W))
    if hot > 0:
        mask = rng.uniform(size=(H, W)) < hot
        var[mask] *= 50.0
    return offset, gain, var


def make_stack(name="stack512", T=None, device="cuda", seed=1234, pixel=0.1, NA=1.4,
               wavelength=0.7, **overrides):
    """Build a named workload.  Returns a dict with ``images`` [T,H,W] and
    ``gamma`` [H,W] (float32 torch tensors on ``device``), ``mask`` (centred
    16x16 numpy), ``alpha``, ``max_iters`` and the generating parameters.
    ``overrides`` replace workload fields (H, W, chains, bg, hot, photons);
    ``photons=(lo, hi)`` draws each emitter's photon count from U(lo, hi)."""
    cfg = dict(WORKLOADS[name])
    if T is not None:
        cfg["T"] = int(T)
    for k, v in overrides.items():
        if k not in cfg:
            raise KeyError("unknown workload field %r" % (k,))
        cfg[k] = v
    rng = numpy.random.default_rng(seed)
    H, W = cfg["H"], cfg["W"]
    field = max(H, W) * pixel
    em = wlc_emitters(cfg["chains"], field, rng) / pixel
    sigma_px = 0.21 * wavelength / NA / pixel
    photons = cfg["photons"]
    if isinstance(photons, (tuple, list)):
        photons = rng.uniform(photons[0], photons[1], size=len(em))
    ideal = render(em, H, W, sigma_px, photons, cfg["bg"])
    offset, gain, var = camera_maps(H, W, rng, cfg["hot"])
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed + 1)
    t_ideal = torch.as_tensor(ideal, dtype=torch.float32, device=dev)
    t_gain = torch.as_tensor(gain, dtype=torch.float32, device=dev)
    t_off = torch.as_tensor(offset, dtype=torch.float32, device=dev)
    t_sd = torch.as_tensor(numpy.sqrt(var), dtype=torch.float32, device=dev)
    images = torch.empty((cfg["T"], H, W), dtype=torch.float32, device=dev)
    chunk = max(1, (1 << 26) // (H * W))
    for f0 in range(0, cfg["T"], chunk):
        n = min(chunk, cfg["T"] - f0)
        lam = t_ideal.expand(n, H, W).contiguous()
        phot = torch.poisson(lam, generator=g)
        adu = phot * t_gain + t_sd * torch.randn((n, H, W), generator=g, device=dev) + t_off
        d = (adu - t_off) / t_gain
        images[f0:f0 + n] = torch.where(d <= 0, torch.full_like(d, 1e-6), d)
    gamma = torch.as_tensor(var / gain ** 2, dtype=torch.float32, device=dev)
    mask = otf_weighted_mask(16, pixel, NA, wavelength)
    return dict(images=images, gamma=gamma, mask=mask, alpha=cfg["alpha"],
                max_iters=cfg["max_iters"], ideal=ideal, name=name, seed=seed, cfg=cfg)


def beads(n, field, rng):
    """Positions (x, y) of n sparse point emitters, uniform over the field."""
    return rng.uniform(0.0, field, size=(n, 2))


def make_mixed(n_stacks=64, seed=4242, device="cuda", sides=(64, 128, 256, 512, 1024, 2048),
               frames=(10, 200), pixel=0.1):
    """The mixed-workload batch: ``n_stacks`` stacks with ROI sides drawn from
    ``sides`` and frame counts U{frames}, each with its own alpha U(0.05, 0.5),
    NA in {1.2, 1.4, 1.49} and wavelength in {520, 600, 700} nm (hence its own
    OTF-weighted mask), and either worm-like chains (100 photons per emitter,
    12 chains per 512 x 512 field) or sparse beads (Gaussian spots of 2000
    photons, 0.05 per um^2); background 10 photons/px and the camera model of
    ``camera_maps``.  Returns a list of dicts as ``make_stack`` does."""
    rng = numpy.random.default_rng(seed)
    dev = torch.device(device)
    out = []
    for k in range(n_stacks):
        side = int(rng.choice(sides))
        T = int(rng.integers(frames[0], frames[1] + 1))
        alpha = float(rng.uniform(0.05, 0.5))
        NA = float(rng.choice([1.2, 1.4, 1.49]))
        wl = float(rng.choice([0.52, 0.6, 0.7]))
        kind = "chains" if rng.uniform() < 0.5 else "beads"
        field = side * pixel
        sigma_px = 0.21 * wl / NA / pixel
        if kind == "chains":
            n_ch = max(1, int(round(12.0 * side * side / (512.0 * 512.0))))
            ideal = render(wlc_emitters(n_ch, field, rng) / pixel, side, side, sigma_px, 100.0,
                           10.0)
        else:
            n_b = max(1, int(round(0.05 * field * field)))
            ideal = render(beads(n_b, field, rng) / pixel, side, side, sigma_px, 2000.0, 10.0)
        offset, gain, var = camera_maps(side, side, rng)
        g = torch.Generator(device=dev)
        g.manual_seed(seed * 1000 + k)
        t_ideal = torch.as_tensor(ideal, dtype=torch.float32, device=dev)
        t_gain = torch.as_tensor(gain, dtype=torch.float32, device=dev)
        t_off = torch.as_tensor(offset, dtype=torch.float32, device=dev)
        t_sd = torch.as_tensor(numpy.sqrt(var), dtype=torch.float32, device=dev)
        images = torch.empty((T, side, side), dtype=torch.float32, device=dev)
        chunk = max(1, (1 << 26) // (side * side))
        for f0 in range(0, T, chunk):
            n = min(chunk, T - f0)
            phot = torch.poisson(t_ideal.expand(n, side, side).contiguous(), generator=g)
            adu = phot * t_gain + t_sd * torch.randn((n, side, side), generator=g,
                                                     device=dev) + t_off
            d = (adu - t_off) / t_gain
            images[f0:f0 + n] = torch.where(d <= 0, torch.full_like(d, 1e-6), d)
        gamma = torch.as_tensor(var / gain ** 2, dtype=torch.float32, device=dev)
        out.append(dict(images=images, gamma=gamma, mask=otf_weighted_mask(16, pixel, NA, wl),
                        alpha=alpha, NA=NA, wavelength=wl, kind=kind, side=side, T=T,
                        name="mixed[%d]" % k))
    return out


# ---- the same physics on the GPU (libncs_b200 ncsb_sim_*) --------------------

_CELL = 8


def render_gpu(emitters_px, H, W, sigma_px, photons, bg, half=5, device="cuda"):
    """``render`` on the device: [H, W] float32 tensor.  Emitters farther than
    ``half`` pixels outside the frame cannot contribute and are dropped; the
    rest are sorted by 8 x 8-pixel cell for the kernel's fixed-order gather."""
    import ctypes
    from . import _lib
    em = numpy.asarray(emitters_px, dtype=numpy.float64).reshape(-1, 2)
    ph = numpy.broadcast_to(numpy.asarray(photons, dtype=numpy.float64), (len(em),))
    fx, fy = numpy.floor(em[:, 0]), numpy.floor(em[:, 1])
    keep = (fx >= -half) & (fx <= W - 1 + half) & (fy >= -half) & (fy <= H - 1 + half)
    em, ph, fx, fy = em[keep], ph[keep], fx[keep], fy[keep]
    ncx, ncy = (W + _CELL - 1) // _CELL, (H + _CELL - 1) // _CELL
    cx = numpy.clip(fx // _CELL, 0, ncx - 1).astype(numpy.int64)
    cy = numpy.clip(fy // _CELL, 0, ncy - 1).astype(numpy.int64)
    cell = cy * ncx + cx
    order = numpy.argsort(cell, kind="stable")
    start = numpy.zeros(ncx * ncy + 1, dtype=numpy.int32)
    numpy.cumsum(numpy.bincount(cell, minlength=ncx * ncy), out=start[1:])
    packed = numpy.stack([em[order, 0], em[order, 1], ph[order]], axis=1).astype(numpy.float32)
    dev = torch.device(device)
    t_em = torch.as_tensor(packed.reshape(-1), device=dev)
    t_start = torch.as_tensor(start, device=dev)
    ideal = torch.empty((H, W), dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        rc = _lib.load().ncsb_sim_render(
            ctypes.c_void_p(t_em.data_ptr() if len(packed) else 0),
            ctypes.c_void_p(t_start.data_ptr()), H, W, float(sigma_px), int(half), float(bg),
            ctypes.c_void_p(ideal.data_ptr()),
            ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    if rc != _lib.NCSB_OK:
        raise RuntimeError("ncsb_sim_render failed with code %d" % rc)
    return ideal


def camera_gpu(ideal, T, offset, gain, var, seed, adu=False, photons=True):
    """T camera frames of ``ideal`` on its device: returns (photo-electrons,
    ADU), each [T, H, W] float32 or None as requested."""
    import ctypes
    from . import _lib
    H, W = ideal.shape
    dev = ideal.device
    maps = [torch.as_tensor(numpy.asarray(m), dtype=torch.float32, device=dev).contiguous()
            for m in (offset, gain, var)]
    ph = torch.empty((T, H, W), dtype=torch.float32, device=dev) if photons else None
    ad = torch.empty((T, H, W), dtype=torch.float32, device=dev) if adu else None
    vp = lambda t: ctypes.c_void_p(t.data_ptr() if t is not None else 0)
    with torch.cuda.device(dev):
        rc = _lib.load().ncsb_sim_camera(
            vp(ideal.contiguous()), T, H, W, vp(maps[0]), vp(maps[1]), vp(maps[2]),
            int(seed) & 0xFFFFFFFFFFFFFFFF, vp(ad), vp(ph),
            ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    if rc != _lib.NCSB_OK:
        raise RuntimeError("ncsb_sim_camera failed with code %d" % rc)
    return ph, ad


def make_stack_gpu(name="stack512", T=None, device="cuda", seed=1234, pixel=0.1, NA=1.4,
                   wavelength=0.7, adu=False, **overrides):
    """``make_stack`` with the rendering and the camera on the GPU (the
    emitter positions, photon counts and camera maps are still drawn on the
    host from the same numpy seed).  With ``adu`` the raw frames and the
    calibration maps are returned too (keys adu, offset, gain, var)."""
    cfg = dict(WORKLOADS[name])
    if T is not None:
        cfg["T"] = int(T)
    for k, v in overrides.items():
        if k not in cfg:
            raise KeyError("unknown workload field %r" % (k,))
        cfg[k] = v
    rng = numpy.random.default_rng(seed)
    H, W = cfg["H"], cfg["W"]
    field = max(H, W) * pixel
    em = wlc_emitters(cfg["chains"], field, rng) / pixel
    sigma_px = 0.21 * wavelength / NA / pixel
    photons = cfg["photons"]
    if isinstance(photons, (tuple, list)):
        photons = rng.uniform(photons[0], photons[1], size=len(em))
    offset, gain, var = camera_maps(H, W, rng, cfg["hot"])
    dev = torch.device(device)
    ideal = render_gpu(em, H, W, sigma_px, photons, cfg["bg"], device=dev)
    phot, raw = camera_gpu(ideal, cfg["T"], offset, gain, var, seed, adu=adu)
    out = dict(images=phot, gamma=torch.as_tensor(var / gain ** 2, dtype=torch.float32, device=dev),
               mask=otf_weighted_mask(16, pixel, NA, wavelength), alpha=cfg["alpha"],
               max_iters=cfg["max_iters"], ideal=ideal, name=name, seed=seed, cfg=cfg)
    if adu:
        out.update(adu=raw,
                   offset=torch.as_tensor(offset, dtype=torch.float32, device=dev),
                   gain=torch.as_tensor(gain, dtype=torch.float32, device=dev),
                   var=torch.as_tensor(var, dtype=torch.float32, device=dev))
    return out


def ideal_image_gpu(xcor, ycor, R, pixelsize=0.1, zoom=8, NA=1.4, wavelength=0.7,
                    device="cuda"):
    """The reference simulator's normalised ideal image (genidealimage,
    python3-6/pyNCS/denoisetools.py:150-186) on the GPU: chain coordinates
    (e.g. the worm-like chains of the reference's randwlcposition.mat)
    shifted to 0, rounded and scaled onto the fine grid of (R zoom)^2 pixels
    (host, as the reference), then occupancy, convolution with the central
    2 Ri x 2 Ri (Ri = 5 zoom // 2) of the device genpsfparam PSF and binning
    (ncsb_sim_ideal_image).  Returns a float32 [R, R] tensor."""
    import ctypes
    from . import _lib
    from .otf import device_psf
    sz = int(R) * int(zoom)
    xco = numpy.round(numpy.asarray(xcor, float) - numpy.min(xcor))
    yco = numpy.round(numpy.asarray(ycor, float) - numpy.min(ycor))
    scale = max(xco.max(), yco.max()) / sz
    xs = torch.as_tensor(xco / scale, dtype=torch.float32, device=device)
    ys = torch.as_tensor(yco / scale, dtype=torch.float32, device=device)
    psf = device_psf(sz, pixelsize / zoom, NA, wavelength, device=device)[0]
    cc, ri = sz // 2, int(zoom) * 5 // 2
    kernel = psf[cc - ri:cc + ri, cc - ri:cc + ri].contiguous()
    fine = torch.empty((sz, sz), dtype=torch.float32, device=device)
    out = torch.empty((R, R), dtype=torch.float32, device=device)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    with torch.cuda.device(out.device):
        rc = _lib.load().ncsb_sim_ideal_image(
            vp(xs), vp(ys), int(xs.numel()), int(R), int(zoom), vp(kernel), 2 * ri, vp(fine),
            vp(out), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    if rc != _lib.NCSB_OK:
        raise RuntimeError("ncsb_sim_ideal_image failed with code %d" % rc)
    return out
