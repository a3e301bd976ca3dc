"""ctypes bindings for the compiled CPU oracle -- TEST INFRASTRUCTURE ONLY.

Mirrors the reference's Python wrapper ``clib/pyCNCS/ncs_c.py``:
  * ``NCSCSubRegion`` (ncs_c.py:67-236) over the reference ``ncsSR*`` ABI,
  * ``cReduceNoise`` (ncs_c.py:250-276) over ``ncsReduceNoise`` (ncs.c:41-147),
  * ``pyReduceNoise`` (ncs_c.py:279-322), the Python-side tiling,
  * ``checkOTFMask`` (ncs_c.py:239-247).
The reference library (``_ref/libncs.so``) is preferred; ``port=True`` or its
absence selects our C restatement (``lib/libncs_port.so``), which exposes the
same whole-image and per-tile operations under ``ncsp_*`` names.
"""
import ctypes
import os
import subprocess

import numpy
from numpy.ctypeslib import ndpointer

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libncs.so")
PORT_LIB = os.path.join(HERE, "lib", "libncs_port.so")

_f64 = ndpointer(dtype=numpy.float64, flags="C_CONTIGUOUS")


class NCSCException(Exception):
    pass


def build(ref_root=None):
    """Compile the oracle libraries: the C port always, the reference's own
    ncs.c and CUDA kernel only when ``ref_root`` names a reference tree."""
    cmd = ["make", "-s", "-C", HERE]
    if ref_root:
        cmd.append("REF=" + ref_root)
    subprocess.run(cmd, check=True)


def _common(lib):
    lib.ncs_oracle_set_overrides.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                             ctypes.c_int]
    lib.ncs_oracle_reset_stats.argtypes = []
    lib.ncs_oracle_get_stats.argtypes = [ctypes.POINTER(ctypes.c_long)] * 4 + \
        [ctypes.POINTER(ctypes.c_int)] * 2
    return lib


_cache = {}


def load_ref():
    """The reference ``ncs.c`` built by ``oracle/Makefile`` (None if absent)."""
    if "ref" not in _cache:
        if not os.path.exists(REF_LIB):
            _cache["ref"] = None
        else:
            lib = _common(ctypes.CDLL(REF_LIB))
            lib.ncsReduceNoise.argtypes = [_f64, _f64, _f64, _f64, ctypes.c_double,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_int]
            lib.ncsReduceNoise.restype = None
            lib.ncsSRCalcLLGradient.argtypes = [ctypes.c_void_p, _f64]
            lib.ncsSRCalcLogLikelihood.argtypes = [ctypes.c_void_p]
            lib.ncsSRCalcLogLikelihood.restype = ctypes.c_double
            lib.ncsSRCalcNCGradient.argtypes = [ctypes.c_void_p, _f64]
            lib.ncsSRCalcNoiseContribution.argtypes = [ctypes.c_void_p]
            lib.ncsSRCalcNoiseContribution.restype = ctypes.c_double
            lib.ncsSRCleanup.argtypes = [ctypes.c_void_p]
            lib.ncsSRGetU.argtypes = [ctypes.c_void_p, _f64]
            lib.ncsSRInitialize.argtypes = [ctypes.c_int]
            lib.ncsSRInitialize.restype = ctypes.c_void_p
            lib.ncsSRNewRegion.argtypes = [ctypes.c_void_p, _f64, _f64]
            lib.ncsSRSetOTFMask.argtypes = [ctypes.c_void_p, _f64]
            lib.ncsSRSetU.argtypes = [ctypes.c_void_p, _f64]
            lib.ncsSRSolve.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
            lib.ncsSRSolve.restype = ctypes.c_int
            _cache["ref"] = lib
    return _cache["ref"]


def load_port():
    """Our C restatement of ``ncs.c`` (built from committed sources)."""
    if "port" not in _cache:
        if not os.path.exists(PORT_LIB):
            build()
        lib = _common(ctypes.CDLL(PORT_LIB))
        lib.ncsp_reduce_noise.argtypes = [_f64, _f64, _f64, _f64, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int)]
        lib.ncsp_reduce_noise.restype = ctypes.c_int
        lib.ncsp_solve_tile.argtypes = [_f64, _f64, _f64, _f64, ctypes.c_double, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_double)]
        lib.ncsp_solve_tile.restype = ctypes.c_int
        lib.ncsp_cost.argtypes = [_f64, _f64, _f64, _f64, ctypes.c_double, ctypes.c_int,
                                  ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double)]
        lib.ncsp_cost.restype = ctypes.c_double
        _cache["port"] = lib
    return _cache["port"]


def library(port=False):
    lib = None if port else load_ref()
    return lib if lib is not None else load_port()


def kind(port=False):
    """"reference" when the compiled reference ``ncs.c`` is used, else "port"."""
    return "port" if (port or load_ref() is None) else "reference"


def set_overrides(max_iterations=0, epsilon=-1.0, m=0, linesearch=-1, port=False):
    """libLBFGS parameter overrides for subsequent solves (see lbfgs_api.h)."""
    for lib in {id(library(port)): library(port), id(load_port()): load_port()}.values():
        lib.ncs_oracle_set_overrides(int(max_iterations), float(epsilon), int(m), int(linesearch))


def reset_stats(port=False):
    library(port).ncs_oracle_reset_stats()


def get_stats(port=False):
    v = [ctypes.c_long() for _ in range(4)] + [ctypes.c_int() for _ in range(2)]
    library(port).ncs_oracle_get_stats(*[ctypes.byref(x) for x in v])
    keys = ["calls", "iterations", "evaluations", "failures", "last_status", "last_iterations"]
    return {k: x.value for k, x in zip(keys, v)}


def _c(a):
    return numpy.ascontiguousarray(a, dtype=numpy.float64)


def checkOTFMask(otf_mask):
    """Hermitian-symmetry check of a centred mask (ncs_c.py:239-247)."""
    otf_mask_fft = numpy.fft.ifft2(numpy.fft.fftshift(otf_mask))
    return not (numpy.max(numpy.imag(otf_mask_fft)) > 1.0e-12)


def cReduceNoise(image, gamma, otf_mask_shifted, alpha, strict=True, port=False):
    """Whole-image NCS in C (ncs_c.py:250-276); mask is already fftshifted."""
    if strict:
        if otf_mask_shifted.shape[0] != otf_mask_shifted.shape[1]:
            raise NCSCException("OTF must be square!")
        if (otf_mask_shifted.shape[0] % 2) != 0:
            raise NCSCException("Sub region size must be divisible by 2!")
    r = otf_mask_shifted.shape[0]
    if image.shape[0] + 2 < r or image.shape[1] + 2 < r:
        raise NCSCException("Image is smaller than the sub-region interior.")
    out = numpy.zeros(image.shape, dtype=numpy.float64)
    lib = library(port)
    if lib is load_ref() and not port:
        lib.ncsReduceNoise(out, _c(image), _c(gamma), _c(otf_mask_shifted), float(alpha),
                           image.shape[0], image.shape[1], r)
    else:
        nf = ctypes.c_int(0)
        ret = lib.ncsp_reduce_noise(out, _c(image), _c(gamma), _c(otf_mask_shifted),
                                    float(alpha), image.shape[0], image.shape[1], r,
                                    ctypes.byref(nf))
        if ret != 0:
            raise NCSCException("ncsp_reduce_noise failed")
    return out


def solve_tile(data, gamma, otf_mask_shifted, alpha, port=False):
    """One tile solved from u0 = data; returns (u, lbfgs_status, final_cost)."""
    r = data.shape[0]
    lib = library(port)
    if lib is load_ref() and not port:
        sr = NCSCSubRegion(r, strict=False)
        sr.newRegion(data, gamma)
        sr.setOTFMaskShifted(otf_mask_shifted)
        ret = lib.ncsSRSolve(sr.c_ncs, float(alpha), 0)
        u = sr.getU()
        f = sr.cost(u, alpha)
        sr.cleanup()
        return u, ret, f
    u = numpy.zeros((r, r))
    f = ctypes.c_double()
    ret = lib.ncsp_solve_tile(u, _c(data), _c(gamma), _c(otf_mask_shifted), float(alpha), r,
                              ctypes.byref(f))
    return u, ret, f.value


class NCSCSubRegion:
    """Per-tile solver over the reference ABI (ncs_c.py:67-236)."""

    def __init__(self, r_size=16, strict=True):
        if r_size % 2:
            raise NCSCException("Sub region size must be divisible by 2!")
        self.lib = load_ref()
        if self.lib is None:
            raise NCSCException("reference library not built")
        self.r_size = r_size
        self.strict = strict
        self.c_ncs = self.lib.ncsSRInitialize(r_size)

    def newRegion(self, image, gamma):
        self.image = image
        self.lib.ncsSRNewRegion(self.c_ncs, _c(image), _c(gamma))

    def setOTFMask(self, otf_mask):
        """Centred mask, as ncs_c.py:206-222 (checked, then fftshifted)."""
        if self.strict and not checkOTFMask(otf_mask):
            raise NCSCException("OTF does not have the expected symmetry!")
        self.setOTFMaskShifted(numpy.fft.fftshift(otf_mask))

    def setOTFMaskShifted(self, mask_shifted):
        self.lib.ncsSRSetOTFMask(self.c_ncs, _c(mask_shifted))

    def setU(self, u):
        self.lib.ncsSRSetU(self.c_ncs, _c(u))

    def getU(self):
        u = numpy.zeros((self.r_size, self.r_size))
        self.lib.ncsSRGetU(self.c_ncs, u)
        return u

    def calcLogLikelihood(self):
        return self.lib.ncsSRCalcLogLikelihood(self.c_ncs)

    def calcNoiseContribution(self):
        return self.lib.ncsSRCalcNoiseContribution(self.c_ncs)

    def calcLLGradient(self):
        g = numpy.zeros(self.r_size * self.r_size)
        self.lib.ncsSRCalcLLGradient(self.c_ncs, g)
        return g

    def calcNCGradient(self):
        g = numpy.zeros(self.r_size * self.r_size)
        self.lib.ncsSRCalcNCGradient(self.c_ncs, g)
        return g

    def cost(self, u, alpha):
        self.setU(u)
        return self.calcLogLikelihood() + alpha * self.calcNoiseContribution()

    def cSolve(self, alpha, verbose=False):
        ret = self.lib.ncsSRSolve(self.c_ncs, float(alpha), 0)
        if self.strict and ret != 0:
            raise NCSCException("Solver failed with error code {0:d}!".format(ret))
        return self.getU()

    def cleanup(self):
        if self.c_ncs is not None:
            self.lib.ncsSRCleanup(self.c_ncs)
            self.c_ncs = None


def pyReduceNoise(image, gamma, otf_mask, alpha, strict=True):
    """Python-side tiling over the C per-tile solver (ncs_c.py:279-322); centred mask."""
    r_size = otf_mask.shape[0]
    s_size = r_size - 2
    sr = NCSCSubRegion(r_size=r_size, strict=False)
    sr.setOTFMask(otf_mask)
    pad_image = numpy.pad(image, 1, "edge")
    pad_gamma = numpy.pad(gamma, 1, "edge")
    out = numpy.zeros_like(image, dtype=numpy.float64)
    for i in range(0, pad_image.shape[0], s_size):
        bx = pad_image.shape[0] - r_size if i + r_size > pad_image.shape[0] else i
        for j in range(0, pad_image.shape[1], s_size):
            by = pad_image.shape[1] - r_size if j + r_size > pad_image.shape[1] else j
            sr.newRegion(pad_image[bx:bx + r_size, by:by + r_size],
                         pad_gamma[bx:bx + r_size, by:by + r_size])
            im = sr.cSolve(alpha)
            out[bx:bx + r_size - 2, by:by + r_size - 2] = im[1:-1, 1:-1]
    sr.cleanup()
    return out
