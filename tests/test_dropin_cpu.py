"""CPU tests of the drop-in layer's host logic that needs no GPU: the
failure warning and verbose summary of cuda/pyCUDANCS/ncs.py:131-159, and the
strict-mode mask checks of :183-197 (checkOTFMask, ncs_c.py:239-247)."""
import warnings

import numpy
import pytest


def test_status_report_warns_like_pycudancs(capsys):
    from ncs_b200.ncs import _status_report
    it = numpy.array([3, 5, 7, 9], numpy.int32)
    # all converged: no warning, no failures
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        assert _status_report(numpy.zeros(4, numpy.int32), it, False) == {}
    # only "reached machine precision" (-5): counted, but no warning (ncs.py:134-137)
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        assert _status_report(numpy.array([0, -5, -5, 0]), it, False) == {-5: 2}
    # any other failure: one warning naming every failed sub-region
    with pytest.warns(UserWarning, match="failed on 3 sub-regions"):
        f = _status_report(numpy.array([-2, -5, -4, 0]), it, True)
    assert f == {-5: 1, -4: 1, -2: 1}
    out = capsys.readouterr().out
    assert "Minimum iterations: 3" in out and "Maximum iterations: 9" in out
    assert "Median iterations: 6.000" in out
    assert "failures of type 'Reached maximum iterations'" in out


def test_strict_mask_checks():
    import ncs_b200
    nc = ncs_b200.NCSCUDA()
    with pytest.raises(ncs_b200.NCSCUDAException):
        nc.setOTFMask(numpy.ones((16, 8)))             # not square
    with pytest.raises(ncs_b200.NCSCUDAException):
        nc.setOTFMask(numpy.ones((8, 8)))              # not the tile size
    asym = numpy.zeros((16, 16))
    asym[3, 4] = 1.0
    with pytest.raises(ncs_b200.NCSCUDAException):
        nc.setOTFMask(asym)                            # not Hermitian-symmetric
    assert ncs_b200.checkOTFMask(numpy.ones((16, 16)))
    assert not ncs_b200.checkOTFMask(asym)
    ncs_b200.NCSCUDA(strict=False).setOTFMask(asym)    # strict=False skips the checks
