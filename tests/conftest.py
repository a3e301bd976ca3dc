import os
import sys

import numpy
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle_libs():
    """Build the CPU oracle once (port always; the reference when its source exists)."""
    from oracle import pycncs
    pycncs.build()
    return pycncs


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


def create_otf_mask_shifted():
    """Gaussian high-pass test mask of opencl/pyOpenCLNCS/py_ref.py:129-137
    (fftshifted, float32), restated here so GPU machines need no reference tree."""
    x = (numpy.arange(16) - 8.0) / 3.0
    gx = numpy.exp(-x * x)
    rc = 1.0 - numpy.outer(gx, gx)
    rc = rc - rc.min()
    rc = rc / rc.max()
    return numpy.fft.fftshift(rc).astype(numpy.float32)


def random_otf_mask(size, rng):
    """Random symmetric mask of clib/pyCNCS/test/py_ref.py:77-85 (centred)."""
    psf = rng.uniform(0.0, 1.0, size=(size, size))
    m = numpy.real(numpy.fft.fftshift(numpy.fft.fft2(psf)))
    m = m - m.min()
    return m / m.max()
