"""CPU tests of oracle/refgpu.py's host side: the tiling with which the GPU
tests and the benchmark drive the reference CUDA kernel.

refgpu cuts tiles as cuda/pyCUDANCS/ncs.py:81-98 does (origins
range(0, H + 2, 14), the last ones moved back to end at the padded edge,
repeats kept) and stitches them as :161-169 does (later tiles overwrite).
The numpy oracle (oracle/numpy_ref.py) follows clib/pyCNCS/ncs.c:66-130,
whose origins are the same without the repeats.  Both must give the same
tiles and the same stitched frames.
"""
import numpy
import pytest
import torch


@pytest.mark.parametrize("H,W", [(512, 512), (70, 61), (27, 29), (14, 14), (30, 19)])
def test_segmentation_matches_the_numpy_oracle(H, W):
    from oracle import numpy_ref as nr
    from oracle import refgpu
    rng = numpy.random.default_rng(H * 1000 + W)
    x = rng.uniform(1.0, 50.0, size=(2, H, W)).astype(numpy.float32)
    g = rng.uniform(2.0, 4.0, size=(H, W)).astype(numpy.float32)
    dt, gt = refgpu.segment(torch.from_numpy(x), torch.from_numpy(g))
    # pyCUDANCS's tile count: every origin of range(0, H + 2, 14), repeats included
    nx, ny = len(range(0, H + 2, 14)), len(range(0, W + 2, 14))
    assert dt.shape == (2 * nx * ny, 16, 16) and gt.shape == dt.shape
    # each distinct tile equals the numpy oracle's tile at the same origin
    d_np, g_np, meta = nr.segment(x, g)
    ox, oy = refgpu.origins(H), refgpu.origins(W)
    by_origin = {(int(f), int(a), int(b)): k for k, (f, a, b) in enumerate(meta)}
    for k in range(dt.shape[0]):
        f, rem = divmod(k, nx * ny)
        i, j = divmod(rem, ny)
        m = by_origin[(f, ox[i], oy[j])]
        assert numpy.array_equal(dt[k].numpy(), d_np[m].astype(numpy.float32))
        assert numpy.array_equal(gt[k].numpy(), g_np[m].astype(numpy.float32))
    # stitching the tiles back gives the frames (later tiles overwrite)
    assert torch.equal(refgpu.stitch(dt, x.shape), torch.from_numpy(x))
    out_np = nr.stitch(d_np, meta, x.shape)
    assert numpy.array_equal(refgpu.stitch(dt, x.shape).numpy(), out_np.astype(numpy.float32))


def test_origins_repeat_where_pycudancs_repeats_them():
    from oracle import refgpu
    # H + 2 = 29: i = 14 and i = 28 both overrun and both move back to 13
    assert refgpu.origins(27) == [0, 13, 13]
    assert refgpu.origins(512)[-2:] == [490, 498]
    assert refgpu.origins(14) == [0, 0]
