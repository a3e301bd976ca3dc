"""GPU tests of the batched launch (ncsb_batch_set / ncsb_batch_reduce_noise):
many stacks with their own shape, alpha and OTF mask in one persistent
launch.

The batched kernel reads each tile's stack descriptor instead of kernel
parameters and otherwise runs the single-stack arithmetic, so every stack's
result, per-tile iterations, status and cost must equal (bit for bit) a
single-stack solve with that stack's alpha and mask.  Also: proposals from
the batched network inference (FP32 and tensor-core) equal the per-stack
ones, the launch can be captured in a CUDA graph and replayed, and bad
batches are refused.
"""
import numpy
import pytest
import torch

from conftest import random_otf_mask

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ncs(cuda_ok):
    import ncs_b200
    return ncs_b200


def odd_stacks(seed=3):
    """Small stacks of awkward shapes, random masks and alphas, one with a
    per-frame gamma map."""
    rng = numpy.random.default_rng(seed)
    shapes = [(2, 14, 14), (3, 37, 53), (1, 64, 64), (2, 95, 130), (1, 16, 200)]
    out = []
    for k, (T, H, W) in enumerate(shapes):
        images = rng.uniform(1.0, 90.0, size=(T, H, W)).astype(numpy.float32)
        if k == 3:
            gamma = rng.uniform(0.5, 30.0, size=(T, H, W)).astype(numpy.float32)
        else:
            gamma = rng.uniform(0.5, 30.0, size=(H, W)).astype(numpy.float32)
        out.append(dict(images=torch.from_numpy(images).cuda(),
                        gamma=torch.from_numpy(gamma).cuda(),
                        mask=random_otf_mask(16, rng), alpha=float(rng.uniform(0.05, 0.5))))
    return out


@pytest.fixture(scope="module")
def stacks(cuda_ok):
    from ncs_b200 import sim
    mixed = sim.make_mixed(6, seed=77, sides=(64, 128, 256), frames=(2, 6))
    return odd_stacks() + mixed


def single_solves(ncs, stacks, **kw):
    outs, stats = [], []
    for st in stacks:
        s = ncs.Solver(alpha=st["alpha"], **kw)
        s.set_otf_mask(st["mask"])
        o, it, status, cost, ev = s.reduce_noise(st["images"], st["gamma"], tile_stats="all")
        outs.append(o)
        stats.append((it, status, cost, ev))
        s.close()
    return outs, [torch.cat([x[i] for x in stats]) for i in range(4)]


def test_batch_equals_single_stack_solves(ncs, stacks):
    ref_out, (it, st, cost, ev) = single_solves(ncs, stacks, max_iters=50)
    s = ncs.Solver(max_iters=50)
    outs = s.batch_set(stacks)
    assert s.batch_tiles == it.numel()
    stats = s.batch_stats()
    s.batch_reduce_noise(stats=stats)
    torch.cuda.synchronize()
    for o, r in zip(outs, ref_out):
        assert torch.equal(o, r)
    assert torch.equal(stats["iters"], it) and torch.equal(stats["status"], st)
    assert torch.equal(stats["cost"], cost) and torch.equal(stats["evals"], ev)


def test_batch_of_one_and_repeat_launches(ncs, stacks):
    st = stacks[1]
    ref, (it, _, _, _) = single_solves(ncs, [st])
    s = ncs.Solver()
    out, = s.batch_set([st])
    for _ in range(2):  # the counter is reset by every launch
        out.zero_()
        stats = s.batch_stats()
        s.batch_reduce_noise(stats=stats)
        torch.cuda.synchronize()
        assert torch.equal(out, ref[0]) and torch.equal(stats["iters"], it)


def test_batch_proposals_and_warm_solve(ncs, stacks):
    from ncs_b200 import warmstart
    net = warmstart.WarmStartNet(seed=3)
    # a non-trivial network: perturb the zero last layer
    wo, nw, bo, nb = warmstart.layer_offsets()[3]
    g = torch.Generator(device="cpu").manual_seed(0)
    net.params[wo:wo + nw] = (0.02 * torch.randn(nw, generator=g)).cuda()
    s = ncs.Solver()
    outs = s.batch_set(stacks)
    u0 = net.propose_batch(s)
    per = torch.cat([net.propose_stack(st["images"], st["gamma"]) for st in stacks])
    assert torch.equal(u0, per)
    stats = s.batch_stats()
    s.batch_reduce_noise(u0_tiles=u0, stats=stats)
    torch.cuda.synchronize()
    off = 0
    for st, o in zip(stacks, outs):
        ss = ncs.Solver(alpha=st["alpha"])
        ss.set_otf_mask(st["mask"])
        n = ss.num_tiles(*st["images"].shape)
        ro, rit, rst, rc, rev, rfb = ss.reduce_noise_from(st["images"], st["gamma"],
                                                          u0[off:off + n].contiguous())
        assert torch.equal(o, ro)
        assert torch.equal(stats["iters"][off:off + n], rit)
        assert torch.equal(stats["start"][off:off + n], rfb)
        off += n
        ss.close()


@pytest.mark.parametrize("fp8", [False, True])
def test_batch_tensor_core_proposals_equal_per_stack(ncs, stacks, fp8):
    """The tensor-core inference over a batch (BF16 or E4M3 operands) reads
    each tile's stack descriptor and otherwise runs the per-stack arithmetic:
    equal bit for bit."""
    from ncs_b200 import warmstart
    net = warmstart.WarmStartNet.load()
    s = ncs.Solver()
    s.batch_set(stacks)
    u0, status = net.propose_batch_tc(s, fp8=fp8)
    per = []
    for st in stacks:
        u, st_status = net.propose_stack_tc(st["images"], st["gamma"], fp8=fp8)
        assert int(st_status.item()) == 0
        per.append(u)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    assert u0.shape[0] == s.batch_tiles
    assert torch.equal(u0, torch.cat(per))


def test_warm_batch_replays_from_a_cuda_graph(ncs, stacks):
    """Tensor-core proposals over the batch and the batched solve from them,
    captured together in one CUDA graph (the mixed workload's launch), replay
    bit for bit like the eager calls."""
    from ncs_b200 import warmstart
    net = warmstart.WarmStartNet.load()
    s = ncs.Solver()
    outs = s.batch_set(stacks)
    u0 = torch.empty((s.batch_tiles, 16, 16), dtype=torch.float32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    stats = s.batch_stats()
    net.propose_batch_tc(s, out=u0, status=st)
    s.batch_reduce_noise(u0_tiles=u0, stats=stats)
    torch.cuda.synchronize()
    ref_u0, ref = u0.clone(), [o.clone() for o in outs]
    ref_it, ref_start = stats["iters"].clone(), stats["start"].clone()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        net.propose_batch_tc(s, out=u0, status=st)
        s.batch_reduce_noise(u0_tiles=u0, stats=stats)
    for _ in range(2):
        u0.zero_()
        for o in outs:
            o.zero_()
        stats["iters"].zero_()
        graph.replay()
        torch.cuda.synchronize()
        assert int(st.item()) == 0
        assert torch.equal(u0, ref_u0)
        for o, r in zip(outs, ref):
            assert torch.equal(o, r)
        assert torch.equal(stats["iters"], ref_it) and torch.equal(stats["start"], ref_start)
    del graph


def test_batch_launch_replays_from_a_cuda_graph(ncs, stacks):
    s = ncs.Solver()
    outs = s.batch_set(stacks)
    stats = s.batch_stats()
    s.batch_reduce_noise(stats=stats)
    torch.cuda.synchronize()
    ref = [o.clone() for o in outs]
    ref_it = stats["iters"].clone()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        s.batch_reduce_noise(stats=stats)
    for o in outs:
        o.zero_()
    stats["iters"].zero_()
    for _ in range(2):
        graph.replay()
    torch.cuda.synchronize()
    for o, r in zip(outs, ref):
        assert torch.equal(o, r)
    assert torch.equal(stats["iters"], ref_it)
    del graph


def test_batch_errors(ncs, stacks):
    s = ncs.Solver()
    with pytest.raises(RuntimeError):
        s.batch_reduce_noise()                     # nothing registered
    bad = dict(stacks[0])
    bad["images"] = torch.zeros((1, 13, 20), device="cuda")
    bad["gamma"] = torch.ones((13, 20), device="cuda")
    with pytest.raises(ValueError):
        s.batch_set([stacks[1], bad])              # 13 rows: NCSB_ESIZE
    p = ncs.Solver(mode="plain")
    p.batch_set([stacks[1]])
    with pytest.raises(RuntimeError):
        p.batch_reduce_noise()                     # spectral form only


def test_autotuner_picks_a_timed_candidate_and_caches(ncs, stacks, tmp_path):
    from ncs_b200 import tune
    s = ncs.Solver()
    outs = s.batch_set(stacks)
    key = tune.batch_key(s) + "/test"
    cands = ({"ctas_per_sm": 3, "m": 1}, {"ctas_per_sm": 1, "m": 2})
    path = str(tmp_path / "tune.json")
    best, tried = tune.autotune(s, lambda: s.batch_reduce_noise(), key, candidates=cands,
                                path=path)
    assert best in cands and len(tried) == 2
    assert best == min(tried, key=lambda x: x[0])[1]
    assert (s.params.ctas_per_sm, s.params.m) == (best["ctas_per_sm"], best["m"])
    # whichever candidate wins, the stopping rule is the same: every tile converges
    stats = s.batch_stats()
    s.batch_reduce_noise(stats=stats)
    torch.cuda.synchronize()
    assert (stats["status"] == 0).all()
    # cached: a second call returns the stored choice without timing
    best2, _ = tune.autotune(s, lambda: 1 / 0, key, candidates=cands, path=path)
    assert best2 == best
