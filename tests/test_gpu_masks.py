"""GPU tests of the OTF masks built on the device (ncsb_genfilter and
ncsb_stack.mask_from_optics).

The device masks must equal the reference's own genfilter output
(python3-6/pyNCS/denoisetools.py:227-261, golden vectors generated from it by
tests/golden/make_golden.py) for all three filter types, and the incoherent
type the host restatement in ncs_b200/otf.py; a batch whose masks are built
from optics on the device must solve as the same batch with host masks.
"""
import os

import numpy
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                    "reference_vectors.npz")


@pytest.fixture(scope="module")
def ncs(cuda_ok):
    import ncs_b200
    return ncs_b200


def test_device_genfilter_matches_reference_vectors(ncs):
    from ncs_b200 import otf
    gold = numpy.load(GOLD)
    types = ["pureN", "adjustable", "OTFweighted"]
    m = otf.device_masks([dict(type=t, pixel_size=0.1, NA=1.4, wavelength=0.7) for t in types])
    for t, got in zip(types, m.cpu().numpy()):
        # FP64 on the device, stored as FP32
        assert numpy.abs(got - gold["genfilter_" + t]).max() <= 1e-6, t


def test_device_incoherent_mask_matches_host(ncs):
    from ncs_b200 import otf
    cases = [(0.1, 1.4, 0.7), (0.1, 1.2, 0.52), (0.1, 1.49, 0.6), (0.065, 1.35, 0.54)]
    m = otf.device_masks([dict(type="incoherent", pixel_size=p, NA=n, wavelength=w)
                          for p, n, w in cases])
    for (p, n, w), got in zip(cases, m.cpu().numpy()):
        assert numpy.abs(got - otf.otf_weighted_mask(16, p, n, w)).max() <= 1e-6


def test_bad_optics_rejected(ncs):
    from ncs_b200 import otf
    with pytest.raises(ValueError):
        otf.device_masks([dict(type="OTFweighted", NA=0.0)])
    with pytest.raises(ValueError):
        otf.device_masks([dict(type="adjustable", h=1.5)])


def test_batch_with_device_masks_equals_host_masks(ncs):
    from ncs_b200 import otf, sim
    stacks = sim.make_mixed(5, seed=123, sides=(64, 128), frames=(2, 4))
    host = [dict(images=st["images"], gamma=st["gamma"], alpha=st["alpha"],
                 mask=otf.otf_weighted_mask(16, 0.1, st["NA"], st["wavelength"]))
            for st in stacks]
    dev = [dict(images=st["images"], gamma=st["gamma"], alpha=st["alpha"],
                optics=dict(type="incoherent", pixel_size=0.1, NA=st["NA"],
                            wavelength=st["wavelength"])) for st in stacks]
    a, b = ncs.Solver(), ncs.Solver()
    oa, ob = a.batch_set(host), b.batch_set(dev)
    sa, sb = a.batch_stats(), b.batch_stats()
    a.batch_reduce_noise(stats=sa)
    b.batch_reduce_noise(stats=sb)
    torch.cuda.synchronize()
    # device and host libm may round a mask value differently in its last
    # FP32 bit; the solves then agree to the solver's own tolerance
    for x, y in zip(oa, ob):
        assert ((x - y).abs() / y.abs().clamp(min=1.0)).max().item() <= 1e-4
    assert abs(sa["iters"].double().mean().item() - sb["iters"].double().mean().item()) <= 0.01


def test_device_genpsfparam_matches_reference_vectors(ncs):
    """The reference's own genpsfparam output (tests/golden/genpsfparam_vectors.npz,
    written by make_golden.py from denoisetools.py:103-115) on even and odd grids."""
    from ncs_b200 import otf
    gold = numpy.load(os.path.join(os.path.dirname(GOLD), "genpsfparam_vectors.npz"))
    for R in (16, 32, 33):
        _, px, na, lam = gold["R%d_params" % R]
        psf, pupil, o = (t.cpu().numpy() for t in otf.device_psf(R, px, na, lam))
        assert numpy.allclose(pupil, gold["R%d_pupil" % R], rtol=1e-6, atol=1e-6)
        assert numpy.allclose(psf, gold["R%d_psf" % R], rtol=1e-5, atol=1e-9)
        assert numpy.allclose(o, gold["R%d_otf" % R], rtol=1e-5, atol=1e-7)
