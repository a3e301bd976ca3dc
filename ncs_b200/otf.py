"""OTF masks for the NCS noise term (16 x 16, returned CENTRED, DC at [8, 8];
``numpy.fft.fftshift`` gives the shifted form the solver takes).

* ``otf_weighted_mask`` -- 1 - normalised incoherent OTF of a circular pupil
  inside the cutoff 2 NA / lambda, 1 outside: the high-pass mask of the
  synthetic workloads (the OTF-weighted idea of pyNCS ``genfilter``, with the
  textbook diffraction-limited OTF instead of a raised cosine).
* ``genfilter`` -- the reference's raised-cosine masks, restated from
  python3-6/pyNCS/denoisetools.py:227-261 (types pureN / adjustable /
  OTFweighted), with ``genkspace`` from :96-101.
"""
import numpy


def genkspace(R, pixelsize):
    """|k| grid of an R x R tile in cycles per unit of pixelsize, centred
    (denoisetools.py:96-101)."""
    X, Y = numpy.meshgrid(numpy.arange(-R / 2, R / 2, 1), numpy.arange(-R / 2, R / 2, 1))
    return numpy.sqrt(X ** 2 + Y ** 2) / (R * pixelsize)


def otf_weighted_mask(R=16, pixelsize=0.1, NA=1.4, wavelength=0.7):
    """1 - OTF(|k| / kc) for |k| < kc = 2 NA / lambda, 1 outside, with the
    circular-pupil incoherent OTF (2/pi)(acos(r) - r sqrt(1 - r^2)).
    Lengths in micrometres.  Returns the centred mask (float64)."""
    kr = genkspace(R, pixelsize)
    kc = 2.0 * NA / wavelength
    rho = numpy.clip(kr / kc, 0.0, 1.0)
    otf = (2.0 / numpy.pi) * (numpy.arccos(rho) - rho * numpy.sqrt(1.0 - rho ** 2))
    return numpy.where(kr < kc, 1.0 - otf, 1.0)


def genfilter(R, pixelsize, NA, Lambda, Type="OTFweighted", w=1, h=0.7):
    """Raised-cosine high-pass of pyNCS (denoisetools.py:227-261); centred."""
    kr = genkspace(R, pixelsize)
    kmax = 1.0 / numpy.sqrt(2.0) / pixelsize
    if Type == "pureN":
        beta = 0.2
        T = (1 - beta) * Lambda / 4 / NA
    elif Type == "adjustable":
        w0 = w * NA / Lambda
        beta = numpy.pi / 2 * (kmax / w0 - 1) / (numpy.arccos(1 - 2 * h) + numpy.pi / 2 * (kmax / w0 - 1))
        T = (1 - beta) / w0 / 2
    elif Type == "OTFweighted":
        beta = 1.0
        T = Lambda / 4 / NA / 1.4
    else:
        raise ValueError("unknown filter type %r" % (Type,))
    rc = 0.5 * (1 + numpy.cos(numpy.pi * T / beta * (kr - (1 - beta) / 2 / T)))
    rc[kr < (1 - beta) / 2 / T] = 1
    rc[kr > (1 + beta) / 2 / T] = 0
    return 1 - rc


def shifted(mask_centred):
    return numpy.fft.fftshift(numpy.asarray(mask_centred))


def device_masks(optics_list, device="cuda"):
    """Centred 16 x 16 masks built on the GPU (libncs_b200 ncsb_genfilter),
    one per dict of ``ncs_b200._lib.optics`` keywords (type, pixel_size, NA,
    wavelength, w, h).  Returns a float32 tensor [n, 16, 16] on ``device``."""
    import ctypes
    import torch
    from . import _lib
    n = len(optics_list)
    arr = (_lib.NcsbOptics * max(n, 1))()
    for i, o in enumerate(optics_list):
        arr[i] = _lib.optics(**o)
    out = torch.empty((n, 16, 16), dtype=torch.float32, device=device)
    with torch.cuda.device(out.device):
        rc = _lib.load().ncsb_genfilter(arr, n, ctypes.c_void_p(out.data_ptr()),
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    if rc != _lib.NCSB_OK:
        raise ValueError("ncsb_genfilter failed with code %d (bad optics?)" % rc)
    return out


def genfilter_odd(n, pixelsize, NA, Lambda, Type=None, w=1.0, h=0.7):
    """Masks of the normalised single-pixel variant (odd n, centred): the
    reference's "matlab - single pixel with normalization/genfilter.m":30-62,
    grid -(n-1)/2 .. (n-1)/2, kmax = n / sqrt(2) / (n pixelsize); default type
    T = lambda / 2 / NA / 1.4, beta = 1."""
    r = numpy.arange(n) - (n - 1) / 2.0
    X, Y = numpy.meshgrid(r, r)
    kr = numpy.sqrt(X ** 2 + Y ** 2) / (n * pixelsize)
    kmax = n / numpy.sqrt(2.0) / (n * pixelsize)
    if Type == "pureN":
        beta = 0.2
        T = (1 - beta) * Lambda / 2 / NA
    elif Type == "adjustable":
        w0 = w * NA / Lambda
        beta = numpy.pi / 2 * (kmax / w0 - 1) / (numpy.arccos(1 - 2 * h) + numpy.pi / 2 * (kmax / w0 - 1))
        T = (1 - beta) / w0 / 2
    else:
        beta = 1.0
        T = Lambda / 2 / NA / 1.4
    rc = 0.5 * (1 + numpy.cos(numpy.pi * T / beta * (kr - (1 - beta) / 2 / T)))
    rc[kr < (1 - beta) / 2 / T] = 1
    rc[kr > (1 + beta) / 2 / T] = 0
    return 1 - rc


def normalized_mask(pixelsize=0.1, NA=1.4, Lambda=0.7):
    """The 3 x 3 mask the normalised variant builds by default: genfilter of
    the segment size Rs + 2 = 3 with twice the NA (reducenoise.m, otfsize = 2)."""
    return genfilter_odd(3, pixelsize, 2.0 * NA, Lambda)


def device_psf(R, pixelsize, NA, wavelength, device="cuda"):
    """genpsfparam of the reference (denoisetools.py:103-115) computed on the GPU
    (ncsb_genpsfparam): returns (PSFn, pupil, OTFn), float32 [R, R] tensors."""
    import ctypes
    import torch
    from . import _lib
    outs = [torch.empty((R, R), dtype=torch.float32, device=device) for _ in range(3)]
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    with torch.cuda.device(outs[0].device):
        rc = _lib.load().ncsb_genpsfparam(int(R), float(pixelsize), float(NA), float(wavelength),
                                          vp(outs[0]), vp(outs[1]), vp(outs[2]),
                                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    if rc != _lib.NCSB_OK:
        raise ValueError("ncsb_genpsfparam failed with code %d" % rc)
    return tuple(outs)
