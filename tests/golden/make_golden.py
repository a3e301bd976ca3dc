"""Generate the golden vectors in tests/golden/ from the reference itself.

Run in a container that has the reference tree and the built oracle
(``make -C oracle REF=REFERENCE_ROOT``):

    python tests/golden/make_golden.py REFERENCE_ROOT

Nothing at test time reads the reference tree; tests only read the .npz files
written here.  Sources used (paths in the HuanglabPurdue/NCS tree):
  * clib/pyCNCS/test/py_ref.py     calcLogLikelihood / calcNoiseContribution /
                                   calcCost, finite-difference gradients,
                                   randomOTFMask, ncsSolve (scipy L-BFGS-B)
  * opencl/pyOpenCLNCS/py_ref.py   createOTFMask, ncsReduceNoise (the numpy
                                   mirror of the reference GPU kernel)
  * clib/pyCNCS/ncs_c.py           cReduceNoise / pyReduceNoise, run through
                                   the reference's own Python wrapper over the
                                   reference ncs.c compiled by oracle/Makefile
  * python3-6/pyNCS/denoisetools.py genfilter (all three filter types) and
                                   genpsfparam (genpsfparam_vectors.npz;
                                   ``--psf-only`` writes just that file)
"""
import importlib.util
import os
import sys
import types

import numpy
import scipy.optimize

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(ref):
    clib_ref = load("clib_py_ref", os.path.join(ref, "clib/pyCNCS/test/py_ref.py"))
    ocl_ref = load("ocl_py_ref", os.path.join(ref, "opencl/pyOpenCLNCS/py_ref.py"))
    out = {}

    # -- cost terms and finite-difference gradients (test_sr.py:12-97) ------
    numpy.random.seed(11)
    n = 4
    U = numpy.random.uniform(0.01, 10.0, size=(n, 16, 16))
    D = numpy.random.uniform(0.01, 10.0, size=(n, 16, 16))
    G = numpy.random.uniform(2.0, 4.0, size=(n, 16, 16))
    numpy.random.seed(12)
    masks = numpy.array([clib_ref.randomOTFMask(16) for _ in range(n)])  # centred
    alpha = 0.02
    out.update(cost_u=U, cost_data=D, cost_gamma=G, cost_masks_centred=masks, cost_alpha=alpha)
    out["cost_ll"] = numpy.array([clib_ref.calcLogLikelihood(U[i], D[i], G[i]) for i in range(n)])
    out["cost_nc"] = numpy.array([clib_ref.calcNoiseContribution(U[i], masks[i]) for i in range(n)])
    out["cost_f"] = numpy.array([clib_ref.calcCost(U[i].ravel(), D[i], G[i], masks[i], alpha)
                                 for i in range(n)])
    out["fd_ll_grad"] = numpy.array([clib_ref.calcLLGradient(U[i], D[i], G[i]) for i in range(2)])
    out["fd_nc_grad"] = numpy.array([clib_ref.calcNCGradient(U[i], masks[i]) for i in range(2)])

    # -- randomOTFMask with a fixed legacy seed (py_ref.py:77-85) -------------
    numpy.random.seed(0)
    out["random_mask_seed0"] = clib_ref.randomOTFMask(16)

    # -- solver cross-check setup of test_sr.py:99-128 -----------------------
    # py_ref.ncsSolve passes a 2-D x0, which current scipy rejects; the same
    # call is made with x0 flattened.
    numpy.random.seed(13)
    sD, sG, sM, sU = [], [], [], []
    for _ in range(3):
        g = numpy.random.uniform(2.0, 4.0, size=(16, 16))
        d = numpy.random.uniform(10.0, 20.0, size=(16, 16))
        m = clib_ref.randomOTFMask(16)
        res = scipy.optimize.minimize(clib_ref.calcCost, d.ravel(), args=(d, g, m, 0.02),
                                      method="L-BFGS-B", options={"maxiter": 200})
        sD.append(d); sG.append(g); sM.append(m); sU.append(res.x.reshape(16, 16))
    out.update(solve_data=numpy.array(sD), solve_gamma=numpy.array(sG),
               solve_masks_centred=numpy.array(sM), solve_u_scipy=numpy.array(sU),
               solve_alpha=0.02)

    # -- GPU-algorithm mirror, test_solver.py:31-74 setup ---------------------
    out["create_otf_mask_shifted"] = ocl_ref.createOTFMask().reshape(16, 16)
    numpy.random.seed(1)
    data = numpy.random.uniform(10.0, 20.0, size=(16, 16)).astype(numpy.float32)
    gamma = numpy.random.uniform(2.0, 4.0, size=(16, 16)).astype(numpy.float32)
    ref_u = numpy.zeros(256)
    it = numpy.zeros(1, dtype=numpy.int32)
    st = numpy.zeros(1, dtype=numpy.int32)
    gr, gc = ocl_ref.createUFFTGrad()
    ocl_ref.ncsReduceNoise(gr, gc, data, gamma, ocl_ref.createOTFMask(), ref_u, it, st,
                           numpy.float32(0.1))
    out.update(mirror_data=data, mirror_gamma=gamma, mirror_u=ref_u.reshape(16, 16),
               mirror_iters=it, mirror_status=st, mirror_alpha=0.1)

    # -- whole-image tiling through the reference wrapper (test_im.py) -------
    lib = os.path.join(REPO, "oracle", "_ref", "libncs.so")
    if os.path.exists(lib):
        import ctypes
        pkg = types.ModuleType("pyCNCS")
        pkg.__path__ = [os.path.join(ref, "clib/pyCNCS")]
        sys.modules["pyCNCS"] = pkg
        loadclib = types.ModuleType("pyCNCS.loadclib")
        loadclib.loadNCSCLibrary = lambda: ctypes.cdll.LoadLibrary(lib)
        sys.modules["pyCNCS.loadclib"] = loadclib
        ncs_c = load("pyCNCS.ncs_c", os.path.join(ref, "clib/pyCNCS/ncs_c.py"))
        numpy.random.seed(21)
        im_size, r_size = 30, 10
        gam = numpy.random.uniform(2.0, 4.0, size=(im_size, im_size))
        img = numpy.random.uniform(0.01, 10.0, size=(im_size, im_size))
        om = clib_ref.randomOTFMask(r_size)
        crops = [(0, 0), (3, 7), (11, 11), (5, 0)]
        res_c, res_py = [], []
        for ix, iy in crops:
            res_c.append(ncs_c.cReduceNoise(img[ix:, iy:], gam[ix:, iy:], numpy.fft.fftshift(om),
                                            0.02))
            res_py.append(ncs_c.pyReduceNoise(img[ix:, iy:], gam[ix:, iy:], om, 0.02))
        out.update(im_image=img, im_gamma=gam, im_mask_centred=om, im_crops=numpy.array(crops),
                   im_alpha=0.02, im_r_size=r_size)
        for k, (a, b) in enumerate(zip(res_c, res_py)):
            out["im_c_%d" % k] = a
            out["im_py_%d" % k] = b

    # -- genfilter (denoisetools.py:227-261) ---------------------------------
    dt_src = open(os.path.join(ref, "python3-6/pyNCS/denoisetools.py")).read()
    ns = {}
    start = dt_src.index("def genkspace")
    stop = dt_src.index("def genpsfparam")
    exec("import numpy as np\n" + dt_src[start:stop], ns)
    start = dt_src.index("class filters")
    stop = dt_src.index("def calcost")
    exec(dt_src[start:stop], ns)
    for t in ("pureN", "adjustable", "OTFweighted"):
        out["genfilter_" + t] = ns["genfilter"](16, 0.1, 1.4, 0.7, t)

    numpy.savez_compressed(os.path.join(HERE, "reference_vectors.npz"), **out)
    print("wrote", len(out), "arrays")


def psf_vectors(ref):
    """genpsfparam (denoisetools.py:103-115) for a few grids -> genpsfparam_vectors.npz.
    The module imports plotting and HDF5 packages at the top, so the function is
    taken from its source text with genkspace and run with numpy and
    scipy.fftpack, as the module itself does."""
    import scipy.fftpack
    dt_src = open(os.path.join(ref, "python3-6/pyNCS/denoisetools.py")).read()
    ns = {"ft": scipy.fftpack}
    start = dt_src.index("def genkspace")
    stop = dt_src.index("def SRhist")
    exec("import numpy as np\n" + dt_src[start:stop], ns)
    out = {}
    for R, px, na, lam in ((16, 0.1, 1.4, 0.7), (32, 0.05, 1.2, 0.52), (33, 0.1, 1.49, 0.6)):
        psf, pupil, otf = ns["genpsfparam"](R, px, na, lam)
        key = "R%d" % R
        out[key + "_params"] = numpy.array([R, px, na, lam])
        out[key + "_psf"], out[key + "_pupil"], out[key + "_otf"] = psf, pupil, otf
    numpy.savez_compressed(os.path.join(HERE, "genpsfparam_vectors.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if not args:
        sys.exit("usage: make_golden.py REFERENCE_ROOT [--psf-only]")
    ref_root = args[0]
    if "--psf-only" not in sys.argv:
        main(ref_root)
    psf_vectors(ref_root)
