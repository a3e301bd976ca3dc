"""Generate tests/golden/sim_vectors.npz: ideal images of the reference's own
simulator, python3-6/pyNCS/denoisetools.py genidealimage (:150-186: SRhist
occupancy of the worm-like-chain positions in python3-6/randwlcposition.mat,
convolution with the cropped genpsfparam PSF, binning), for a few grid sizes
and zoom factors.

    python tests/golden/make_sim_golden.py REFERENCE_ROOT

The module imports plotting and HDF5 packages at the top, which are absent
here, so the functions are taken from its source text (genkspace through
genidealimage, and segimg / binimage) and run with numpy and scipy, as the
module itself does.  Written: the chain coordinates read from the .mat file
(so that tests need no reference tree), and per case the ideal image, the
PSF kernel and the occupancy histogram.
"""
import os
import sys

import numpy
import scipy.fftpack
import scipy.io
import scipy.signal

HERE = os.path.dirname(os.path.abspath(__file__))
# (image size R, zoom, pixel size um, NA, wavelength um)
CASES = [(32, 8, 0.1, 1.4, 0.7), (64, 4, 0.1, 1.2, 0.6), (128, 2, 0.1, 1.49, 0.52),
         (48, 1, 0.1, 1.4, 0.7)]


def load_functions(ref):
    src = open(os.path.join(ref, "python3-6/pyNCS/denoisetools.py")).read()
    ns = {"np": numpy, "ft": scipy.fftpack, "sio": scipy.io, "sig": scipy.signal}
    for a, b in (("def segimg", "def padedge"), ("def binimage", "def genkspace"),
                 ("def genkspace", "def cropimage")):
        exec(src[src.index(a):src.index(b)], ns)
    return ns


def main(ref):
    ns = load_functions(ref)
    mat = os.path.join(ref, "python3-6/randwlcposition.mat")
    cor = scipy.io.loadmat(mat)["random_wlc"]
    out = {"xcor": cor[:, 0, :].ravel(), "ycor": cor[:, 1, :].ravel()}
    for R, zoom, px, na, lam in CASES:
        normimg, kernel = ns["genidealimage"](R, px, zoom, na, lam, mat)
        key = "R%d_z%d" % (R, zoom)
        out[key + "_params"] = numpy.array([R, zoom, px, na, lam])
        out[key + "_img"] = normimg
        out[key + "_kernel"] = kernel
    numpy.savez_compressed(os.path.join(HERE, "sim_vectors.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_sim_golden.py REFERENCE_ROOT")
    main(sys.argv[1])
