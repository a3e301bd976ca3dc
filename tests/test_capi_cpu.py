"""CPU tests of the C ABI library: it loads, exports every symbol the header
declares, and its host-only functions agree with the oracle.  No device
compute is called here."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from ncs_b200 import _lib, build
    build.build()
    return _lib.load()


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "ncs_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(ncsb_[a-z_0-9]+)\s*\(", hdr)))


def test_exports_every_declared_symbol(lib):
    from ncs_b200 import _lib
    syms = declared_symbols()
    assert set(syms) == set(_lib.EXPORTS)
    for s in syms:
        assert hasattr(lib, s), s


def test_default_params(lib):
    from ncs_b200 import _lib
    p = _lib.default_params()
    assert (p.alpha, p.max_iters, p.m, p.epsilon, p.c1, p.min_step, p.mode) == \
        (0.2, 200, 1, 1e-5, 1e-4, 1e-6, 2)


def test_num_tiles_matches_oracle(lib):
    from ncs_b200 import _lib
    from oracle import numpy_ref as nr
    for T, H, W in [(1, 256, 256), (200, 512, 512), (100, 2048, 2048), (3, 14, 31), (2, 45, 37)]:
        assert _lib.num_tiles(T, H, W) == T * len(nr.tile_origins(H)) * len(nr.tile_origins(W))
    assert _lib.num_tiles(1, 256, 256) == 361
    assert _lib.num_tiles(200, 512, 512) == 273800
    assert _lib.num_tiles(100, 2048, 2048) == 2160900
    with pytest.raises(ValueError):
        _lib.num_tiles(1, 13, 40)


def test_null_handle_is_rejected(lib):
    from ncs_b200 import _lib
    assert lib.ncsb_set_otf_mask(None, None) == _lib.NCSB_EINVAL
    assert lib.ncsb_destroy(None) == _lib.NCSB_EINVAL
    assert lib.ncsb_reduce_noise(None, None, 1, 16, 16, None, 0, None, None, None, None, None,
                                 None) == _lib.NCSB_EINVAL
    assert lib.ncsb_last_error(None) == b"null handle"
    n = ctypes.c_int64()
    assert lib.ncsb_num_tiles(1, 16, 16, None) == _lib.NCSB_EINVAL
    assert lib.ncsb_num_tiles(-1, 16, 16, ctypes.byref(n)) == _lib.NCSB_EINVAL


def test_stack_descriptor_layout():
    """ctypes mirrors of ncsb_stack (3 pointers, 4 int32, a double, 256
    floats, an int32 flag, ncsb_optics) and ncsb_optics (int32 + 5 doubles),
    with C's alignment of the double members."""
    import ctypes
    from ncs_b200 import _lib
    S = _lib.NcsbStack
    assert ctypes.sizeof(_lib.NcsbOptics) == 48 and _lib.NcsbOptics.pixel_size.offset == 8
    assert S.alpha.offset == 40 and S.mask_shifted.offset == 48
    assert S.mask_from_optics.offset == 1072 and S.optics.offset == 1080
    assert ctypes.sizeof(S) == 1128
    C = _lib.NcsbCalibration
    assert C.n_levels.offset == 24 and C.levels.offset == 28 and ctypes.sizeof(C) == 40


def test_mixed_workload_parameters():
    from ncs_b200 import sim
    st = sim.make_mixed(12, seed=5, device="cpu", sides=(64, 128), frames=(2, 4))
    for s in st:
        T, H, W = s["images"].shape
        assert H == W == s["side"] and H in (64, 128) and 2 <= T <= 4
        assert 0.05 <= s["alpha"] <= 0.5 and s["NA"] in (1.2, 1.4, 1.49)
        assert s["wavelength"] in (0.52, 0.6, 0.7) and s["kind"] in ("chains", "beads")
        assert s["mask"].shape == (16, 16) and (s["images"] > 0).all()
    assert len({(s["NA"], s["wavelength"]) for s in st}) > 1


def test_host_side_rejections_and_empty_calls(lib):
    """Checks the entries make before any device work: a null handle, bad
    shapes and parameters are rejected, and a call for 0 frames succeeds with
    null data buffers (an empty tensor's data_ptr() is 0) without touching a
    device."""
    from ncs_b200 import _lib
    EINVAL, OK, ESIZE = _lib.NCSB_EINVAL, _lib.NCSB_OK, _lib.NCSB_ESIZE
    cal = _lib.NcsbCalibration()
    assert lib.ncsb_reduce_noise_adu_typed(None, None, 1, 1, 16, 16, ctypes.byref(cal), None,
                                           None, None, None, None, None) == EINVAL
    assert lib.ncsb_reduce_noise_adu_host(None, None, 1, 1, 16, 16, ctypes.byref(cal), None,
                                          0, 0, None) == EINVAL
    # the handle-free entries: no-alloc solve and the normalised variant
    p = _lib.default_params()
    mask = (ctypes.c_float * 256)(*([1.0] * 256))
    m3 = (ctypes.c_float * 9)(*([1.0] * 9))
    noalloc, norm = lib.ncsb_reduce_noise_noalloc, lib.ncsb_reduce_noise_normalized
    assert noalloc(ctypes.byref(p), mask, None, 0, 20, 24, None, 0, None,
                   None, None, None, None, None) == OK
    assert noalloc(ctypes.byref(p), mask, None, 1, 20, 24, None, 0, None,
                   None, None, None, None, None) == EINVAL          # data needed for 1 frame
    assert noalloc(ctypes.byref(p), mask, None, 0, 10, 24, None, 0, None,
                   None, None, None, None, None) == ESIZE           # shape still checked
    assert noalloc(None, mask, None, 0, 20, 24, None, 0, None, None, None, None, None,
                   None) == EINVAL
    bad = _lib.default_params()
    bad.m = 0
    assert noalloc(ctypes.byref(bad), mask, None, 0, 20, 24, None, 0, None, None, None, None,
                   None, None) == EINVAL
    assert norm(None, 0, 8, 8, None, 0, m3, 1.0, 15, 1e-6, None, None, None, None, None) == OK
    assert norm(None, 1, 8, 8, None, 0, m3, 1.0, 15, 1e-6, None, None, None, None,
                None) == EINVAL
    assert norm(None, 0, 8, 8, None, 0, m3, -1.0, 15, 1e-6, None, None, None, None,
                None) == EINVAL                                      # negative alpha
    assert norm(None, 0, 8, 8, None, 0, None, 1.0, 15, 1e-6, None, None, None, None,
                None) == EINVAL                                      # no mask
