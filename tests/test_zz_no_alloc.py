"""GPU test of ncsb_reduce_noise_noalloc, the allocation-free entry point.

That entry point serves callers that may not allocate device memory while
they run (a plug-in inside an acquisition or image-server process whose host
application owns the GPU memory through its own pool, or a real-time pipeline
that bans cudaMalloc after start-up because it can synchronise the device);
they cannot create a handle, so the work counter and the mask table live in
a static device array instead.  Here it is called through the C ABI twice in
a row, with different stacks and masks so the second call cannot lean on the
first call's leftovers, and each result must equal what the handle-based
ncsb_reduce_noise returns for the same inputs: the same kernel runs, so
pixels, iteration counts, statuses and costs must agree exactly.

The no-alloc call comes first in each case, so in a fresh process it also
exercises the one-time per-device set-up.  This file is named to be
collected last.
"""
import ctypes

import numpy
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _case(seed, T, H, W):
    from ncs_b200 import otf
    rng = numpy.random.default_rng(seed)
    images = rng.uniform(0.5, 150.0, size=(T, H, W)).astype(numpy.float32)
    gamma = (rng.exponential(15.0, size=(H, W)) + 0.05).astype(numpy.float32)
    na = 1.4 if seed % 2 else 1.2
    mask = numpy.fft.fftshift(otf.otf_weighted_mask(16, 0.1, na, 0.7)).astype(numpy.float32)
    return images, gamma, numpy.ascontiguousarray(mask)


def test_noalloc_matches_handle_entry_point_twice(cuda_ok):
    import ncs_b200
    from ncs_b200 import _lib
    lib = _lib.load()
    cases = [(_case(1, 3, 45, 61), 0.2, 25), (_case(2, 2, 70, 33), 0.35, 40)]
    for (images, gamma, mask), alpha, cap in cases:
        T, H, W = images.shape
        n = _lib.num_tiles(T, H, W)
        x = torch.from_numpy(images).cuda()
        g = torch.from_numpy(gamma).cuda()
        params = _lib.default_params()
        params.alpha = alpha
        params.max_iters = cap
        out = torch.full_like(x, -1.0)
        it = torch.full((n,), -9, dtype=torch.int32, device="cuda")
        st = torch.full((n,), -9, dtype=torch.int32, device="cuda")
        cost = torch.zeros(n, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream()
        rc = lib.ncsb_reduce_noise_noalloc(
            ctypes.byref(params), mask.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), _ptr(x),
            T, H, W, _ptr(g), 0, _ptr(out), _ptr(it), _ptr(st), _ptr(cost), None,
            ctypes.c_void_p(stream.cuda_stream))
        assert rc == _lib.NCSB_OK
        torch.cuda.synchronize()

        s = ncs_b200.Solver(alpha=alpha, max_iters=cap)
        s.set_otf_mask_shifted(mask)
        ref, rit, rst, rcost = s.reduce_noise(x, g, tile_stats=True)
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
        assert torch.equal(it, rit)
        assert torch.equal(st, rst)
        assert torch.equal(cost, rcost)
        assert set(st.cpu().numpy().tolist()) <= {0, -2}
        s.close()


def test_noalloc_rejects_bad_arguments(cuda_ok):
    from ncs_b200 import _lib
    lib = _lib.load()
    params = _lib.default_params()
    mask = numpy.ones((16, 16), dtype=numpy.float32)
    mp = mask.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    x = torch.ones(1, 20, 20, device="cuda")
    o = torch.empty_like(x)
    assert lib.ncsb_reduce_noise_noalloc(None, mp, _ptr(x), 1, 20, 20, _ptr(x), 0, _ptr(o),
                                         None, None, None, None, None) == _lib.NCSB_EINVAL
    small = torch.ones(1, 10, 10, device="cuda")
    assert lib.ncsb_reduce_noise_noalloc(ctypes.byref(params), mp, _ptr(small), 1, 10, 10,
                                         _ptr(small), 0, _ptr(small), None, None, None, None,
                                         None) == _lib.NCSB_ESIZE
    params.m = 99
    assert lib.ncsb_reduce_noise_noalloc(ctypes.byref(params), mp, _ptr(x), 1, 20, 20, _ptr(x),
                                         0, _ptr(o), None, None, None, None,
                                         None) == _lib.NCSB_EINVAL
