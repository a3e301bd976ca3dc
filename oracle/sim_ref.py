"""FP64 restatement of the reference's ideal-image simulator (TEST
INFRASTRUCTURE ONLY: the checker of ncs_b200's device simulator, never
called by the product).

python3-6/pyNCS/denoisetools.py:
  * genkspace / genpsfparam (:96-115): pupil |k| <= NA / lambda on the centred
    grid, PSF = |fftshift(fft2(pupil))|^2 normalised to sum 1;
  * SRhist (:117-148): the emitter positions' occupancy on the fine grid --
    after genidealimage clips the counts at 1 (:177) only whether a fine
    pixel holds a position matters;
  * genidealimage (:150-186): positions shifted to start at 0, rounded, scaled
    so the larger extent spans the fine grid (sz = R zoom), occupancy, 'same'
    convolution with the central 2 Ri x 2 Ri of the PSF (Ri = 5 zoom // 2),
    absolute value, transpose, then (zoom > 1) binimage (:88-94) -- whose
    block ordering transposes again -- divided by zoom;
  * addnoise (:205-213): ideal = |normimg| I + bg, Poisson, x gain, + sqrt(var)
    N(0, 1), + offset; so E[adu] = gain ideal + offset and
    Var[adu] = gain^2 ideal + var.
Pinned to outputs of the reference's own genidealimage
(tests/golden/sim_vectors.npz, written by tests/golden/make_sim_golden.py).
"""
import numpy


def genkspace(R, pixelsize):
    X, Y = numpy.meshgrid(numpy.arange(-R / 2, R / 2, 1), numpy.arange(-R / 2, R / 2, 1))
    return numpy.sqrt(X ** 2 + Y ** 2) / (R * pixelsize)


def genpsfparam(R, pixelsize, NA, wavelength):
    """Normalised PSF (sum 1) of the circular pupil, centred."""
    pupil = genkspace(R, pixelsize)
    pupil[pupil > NA / wavelength] = 0.0
    a = numpy.fft.fftshift(numpy.fft.fft2(pupil))
    psf = (a * a.conj()).real
    return psf / psf.sum()


def occupancy(sz, xs, ys):
    """1 where a fine pixel [floor(x), floor(y)] holds a position (x -> row)."""
    h = numpy.zeros((sz, sz))
    ix, iy = numpy.floor(xs).astype(int), numpy.floor(ys).astype(int)
    ok = (ix >= 0) & (ix < sz) & (iy >= 0) & (iy < sz)
    h[ix[ok], iy[ok]] = 1.0
    return h


def fine_positions(xcor, ycor, sz):
    """Positions on the fine grid: shifted to 0, rounded, scaled so that the
    larger extent is sz (genidealimage's xs, ys)."""
    xco = numpy.round(xcor - xcor.min())
    yco = numpy.round(ycor - ycor.min())
    scale = max(xco.max(), yco.max()) / sz
    return xco / scale, yco / scale


def psf_kernel(R, pixelsize, zoom, NA, wavelength):
    sz = R * zoom
    cc, ri = sz // 2, zoom * 5 // 2
    return genpsfparam(sz, pixelsize / zoom, NA, wavelength)[cc - ri:cc + ri, cc - ri:cc + ri]


def same_conv(img, k):
    """scipy.signal.fftconvolve(img, k, 'same') by direct summation: the full
    convolution's centre, starting at (len(k) - 1) // 2 on each axis."""
    n, m = img.shape
    kh, kw = k.shape
    full = numpy.zeros((n + kh - 1, m + kw - 1))
    for u in range(kh):
        for v in range(kw):
            full[u:u + n, v:v + m] += k[u, v] * img
    a, b = (kh - 1) // 2, (kw - 1) // 2
    return full[a:a + n, b:b + m]


def ideal_image(xcor, ycor, R, pixelsize, zoom, NA, wavelength):
    """genidealimage: the normalised ideal image [R, R] and the PSF kernel."""
    sz = R * zoom
    xs, ys = fine_positions(numpy.asarray(xcor, float), numpy.asarray(ycor, float), sz)
    k = psf_kernel(R, pixelsize, zoom, NA, wavelength)
    conv = numpy.abs(same_conv(occupancy(sz, xs, ys), k))
    if zoom == 1:
        return conv.T, k
    # transpose, then binimage's block sums (which transpose back), / zoom
    return conv.reshape(R, zoom, R, zoom).sum(axis=(1, 3)) / zoom, k


def camera_moments(ideal_photons, gain, var, offset):
    """E and Var of addnoise's ADU for an ideal photon image."""
    return gain * ideal_photons + offset, gain * gain * ideal_photons + var
