"""GPU test of ncsb_reduce_noise_noalloc, the allocation-free entry point.

That entry point serves callers that may not allocate device memory while
they run (a plug-in inside an acquisition or image-server process whose host
application owns the GPU memory through its own pool, or a real-time pipeline
that bans cudaMalloc after start-up because it can synchronise the device);
they cannot create a handle, so the work counter and the mask table live in
a static device array instead.  Here it is called through the C ABI twice in
a row, with different stacks and masks so the second call cannot lean on the
first call's leftovers, in every solver mode and with a fixed CTA count, and
each result must equal what the handle-based ncsb_reduce_noise returns for
the same inputs: the same kernel runs, so pixels, iteration counts, statuses
and costs must agree exactly.  A last case records the call in a CUDA graph
and replays it.

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


def _noalloc(lib, params, mask, x, g, out, it, st, cost, stream):
    from ncs_b200 import _lib
    T, H, W = x.shape
    return lib.ncsb_reduce_noise_noalloc(
        ctypes.byref(params), mask.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), _ptr(x),
        T, H, W, _ptr(g), 0, _ptr(out), _ptr(it), _ptr(st), _ptr(cost), None,
        ctypes.c_void_p(stream.cuda_stream))


# (mode, history size m, resident CTAs per SM; 0 = the library's choice)
MODES = [("spectral", 1, 0), ("plain", 4, 0), ("plain_wg", 4, 0), ("spectral", 2, 3),
         ("plain", 2, 2)]


@pytest.mark.parametrize("mode,m,ctas", MODES)
def test_noalloc_matches_handle_entry_point_twice(cuda_ok, mode, m, ctas):
    import ncs_b200
    from ncs_b200 import _lib
    from ncs_b200.ncs import _MODES
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
        params.mode = _MODES[mode]
        params.m = m
        params.ctas_per_sm = ctas
        out = torch.full_like(x, -1.0)
        it = torch.full((n,), -9, dtype=torch.int32, device="cuda")
        st = torch.full((n,), -9, dtype=torch.int32, device="cuda")
        cost = torch.zeros(n, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream()
        assert _noalloc(lib, params, mask, x, g, out, it, st, cost, stream) == _lib.NCSB_OK
        torch.cuda.synchronize()

        s = ncs_b200.Solver(alpha=alpha, max_iters=cap, mode=mode, m=m, ctas_per_sm=ctas)
        s.set_otf_mask_shifted(mask)
        ref, rit, rst, rcost = s.reduce_noise(x, g, tile_stats=True)
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
        assert torch.equal(it, rit)
        assert torch.equal(st, rst)
        assert torch.equal(cost, rcost)
        assert set(st.cpu().numpy().tolist()) <= {0, -2}
        s.close()


def test_noalloc_captured_in_a_graph_and_replayed(cuda_ok):
    """The call enqueues only kernels (the mask table goes to the device as a
    kernel argument), so it can be recorded in a CUDA graph after its first,
    set-up call; each replay re-initialises the scratch and gives the handle
    entry's result."""
    import ncs_b200
    from ncs_b200 import _lib
    lib = _lib.load()
    images, gamma, mask = _case(3, 2, 40, 52)
    T, H, W = images.shape
    n = _lib.num_tiles(T, H, W)
    x = torch.from_numpy(images).cuda()
    g = torch.from_numpy(gamma).cuda()
    params = _lib.default_params()
    params.max_iters = 30
    out = torch.zeros_like(x)
    it = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    cost = torch.zeros(n, dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):  # set-up call, outside the capture
        assert _noalloc(lib, params, mask, x, g, out, it, st, cost, side) == _lib.NCSB_OK
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        rc = _noalloc(lib, params, mask, x, g, out, it, st, cost,
                      torch.cuda.current_stream())
    assert rc == _lib.NCSB_OK
    s = ncs_b200.Solver(max_iters=30)
    s.set_otf_mask_shifted(mask)
    ref, rit, rst, rcost = s.reduce_noise(x, g, tile_stats=True)
    for _ in range(2):
        out.fill_(-1.0)
        it.fill_(-9)
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
        assert torch.equal(it, rit)
        assert torch.equal(st, rst)
        assert torch.equal(cost, rcost)
    del graph
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
