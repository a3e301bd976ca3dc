#!/usr/bin/env python
"""NCS throughput benchmark on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): ``stack512`` -- 200 frames of 512 x 512 float32 photo-
electrons (worm-like-chain structure, sCMOS camera model, seeded synthetic),
one shared gamma map, OTF-weighted 16x16 mask, alpha 0.2, L-BFGS capped at 20
iterations, all 273,800 tiles in one persistent launch.  A step is one solve
of the whole stack.  Inputs and outputs (210 MB each) exceed the 126 MB L2, so
no flush is needed between steps.

Prints one JSON line.  ``value`` is Mpixel/s of the whole job (all ranks) with
the stack resident in HBM, timed with CUDA events; ``e2e`` is the same metric
through the public ``Solver.reduce_noise_host`` API (the C entry
ncsb_reduce_noise_host) from pinned host memory: every step copies the stack
in, solves it and copies it out, in frame chunks round-robin over four
streams so that the copies overlap the solve.  Under torchrun each rank solves
its own stack (replicas by frame, weak scaling, no collective in the data
path); the time
is the max over ranks.  ``--impl reference`` times the reference's own CPU
path (pyCNCS ncs.c compiled by oracle/Makefile, else the oracle's C port) on
all host cores instead, and beside it, where a GPU and the build are present,
the reference's own CUDA kernel (cuda/ncs.cu compiled unmodified) on the same
workload as ``reference_gpu``.  ``e2e.roofline`` is the host link's measured
ceiling: plain copies of the same bytes in and out at once.
"""
import argparse
import ctypes
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic FP32 work per tile, the roofline numerator.  A real 16x16
# 2-D FFT is counted as 2.5 N log2 N = 5,120 flops (N = 256).
#   start (both forms): Q u by a forward + inverse FFT and the spectrum
#     weighting (11,264), gradient and norms (3,328)              14,592
#   per line-search trial: 256 x (log1p, divide, 6 flops)          2,048
# plain form (scalar initial matrix), per iteration: Q p (11,264),
#   directional dots (1,536), accepted point + gradient (2,304), norms and
#   curvature dots (2,048), plus 2,048 per stored pair (2 dots, 2 axpys)
# spectral form, per iteration: one forward + one inverse FFT, the spectrum
#   weighting and w = q - lambda p (11,776), directional dots (1,536),
#   accepted point + gradient + curvature (2,816), norms and lambda (2,048),
#   plus 2,560 per stored pair (2 dots, 3 axpys)
FLOP_INIT = 11264 + 3328
FLOP_TRIAL = 2048
FLOP_ITER_BASE = {"plain": 11264 + 1536 + 2304 + 2048, "plain_wg": 11264 + 1536 + 2304 + 2048,
                  "spectral": 11776 + 1536 + 2816 + 2048}
FLOP_PER_PAIR = {"plain": 4 * 256 * 2, "plain_wg": 4 * 256 * 2, "spectral": 5 * 256 * 2}
# the tensor-core forms run the spectral algorithm (transforms on the tensor cores)
for _f in ("tc_tf32", "tc_bf16x3"):
    FLOP_ITER_BASE[_f], FLOP_PER_PAIR[_f] = FLOP_ITER_BASE["spectral"], FLOP_PER_PAIR["spectral"]
# Warp instructions per solver pass (one iteration or the initial gradient):
# executed warp instructions / (tiles x passes) from one ncu capture of each
# kernel on stack512 at 64 frames, at the commit named in WARP_INST_MEASURED.
# Used for the issue-rate bound, the one that limits these kernels; a kernel
# changed since that commit needs a new capture.
WARP_INST_PER_PASS = {"spectral": 532251760 / (87616 * 6.047982),
                      "plain": 2130097923 / (87616 * 15.693230),
                      "plain_wg": 7479161369 / (87616 * 15.5538)}
# multiply-adds x 2 of the warm-start network per 16x16 tile:
# 256 px x 9 taps x (2*32 + 32*32 + 32*32 + 32*1)
INFER_FLOP_PER_TILE = 2 * 256 * 9 * (2 * 32 + 32 * 32 + 32 * 32 + 32 * 1)
WARP_INST_MEASURED = {"spectral": "35be777", "plain": "3d152ab", "plain_wg": "cf1c4d5"}
KERNEL = {"plain": "ncs_warp_kernel", "plain_wg": "ncs_plain_kernel",
          "spectral": "ncs_spectral_kernel", "tc_tf32": "ncs_tc_kernel<TF32>",
          "tc_bf16x3": "ncs_tc_kernel<BF16x3>"}
# Tensor-core forms: MMA FLOPs executed per tile and pass (one transform pair),
# from the four GEMM stages over 8 tiles (M = 128): stage 1 N 16 x K 16,
# stages 2 and 3 N 32 x K 32, stage 4 N 16 x K 24 (TF32) or K 32 (BF16); the
# three-way BF16 split runs every product three times.  The algorithmic
# figure of a dense 256 x 256 Q-apply is 2 x 256 x 256 = 131,072 per pass.
TC_EXEC_FLOP_PER_PASS = {
    "tc_tf32": 2 * 128 * (16 * 16 + 2 * 32 * 32 + 16 * 24) // 8,
    "tc_bf16x3": 3 * 2 * 128 * (16 * 16 + 2 * 32 * 32 + 16 * 32) // 8}
DENSE_Q_FLOP_PER_PASS = 2 * 256 * 256


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def fp32_peak_tflops(sm_mhz, n_sms):
    return n_sms * 128 * 2 * sm_mhz * 1e6 / 1e12


class Clocks:
    """nvidia-smi sampling (20 ms period) around the timed region; the samples
    whose timestamps fall inside it are the ones reported."""
    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def start(self):
        """Start sampling; returns once the first sample has been written."""
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        deadline = time.time() + 5.0
        while time.time() < deadline and os.path.getsize(self.path) == 0:
            time.sleep(0.02)

    def begin(self):
        self.t0 = time.time()

    def end(self):
        self.t1 = time.time()

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.05)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 10:
                    try:
                        parts[0] = datetime.datetime.strptime(
                            parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                    except ValueError:
                        continue
                    rows.append(parts)
        os.unlink(self.path)
        inside = rows
        if self.t0 is not None and self.t1 is not None:
            inside = [r for r in rows if self.t0 - 0.02 <= r[0] <= self.t1 + 0.02]
        window = "timed region"
        if not inside:  # region shorter than the sampling period: nearest samples
            inside, window = rows, "sampling run around the timed region"
        if not inside:
            return None
        sm = [float(r[2]) for r in inside if r[2].replace(".", "", 1).isdigit()]
        mx = [float(r[3]) for r in inside if r[3].replace(".", "", 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in inside for i in range(4) if r[6 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(inside), "window": window}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce_device():
    # NCCL reduces device tensors; gloo (CPU-only runs) host tensors
    return "cuda" if torch.cuda.is_available() else "cpu"


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world):
    if world == 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def host_link_ceiling(h_in, h_out, d_res, stream, reps=5):
    """The e2e roofline: plain copies of the same bytes over the host link.
    Times (CUDA events, median of ``reps``) the copy of ``h_in`` to the device
    alone, of the device result ``d_res`` to ``h_out`` alone, and both at once
    on two streams -- the floor for any pipeline that must move the stack in
    and the result out.  Overwrites ``h_out`` with ``d_res``."""
    d_in = torch.empty(h_in.shape, dtype=h_in.dtype, device=d_res.device)
    s_in, s_out = torch.cuda.Stream(d_res.device), torch.cuda.Stream(d_res.device)

    def timed(up, down):
        ms = []
        for _ in range(reps + 1):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            s_in.wait_stream(stream)
            s_out.wait_stream(stream)
            if up:
                with torch.cuda.stream(s_in):
                    d_in.copy_(h_in, non_blocking=True)
            if down:
                with torch.cuda.stream(s_out):
                    h_out.copy_(d_res, non_blocking=True)
            stream.wait_stream(s_in)
            stream.wait_stream(s_out)
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        ms = sorted(ms[1:])
        return ms[len(ms) // 2]

    h2d, d2h, both = timed(True, False), timed(False, True), timed(True, True)
    nb_in, nb_out = h_in.numel() * h_in.element_size(), d_res.numel() * d_res.element_size()
    del d_in
    return {"bound": "host link (PCIe), measured copies of the same bytes",
            "h2d_gbs": nb_in / h2d / 1e6, "d2h_gbs": nb_out / d2h / 1e6,
            "h2d_ms": h2d, "d2h_ms": d2h, "both_ms": both,
            "note": "frac = both_ms / e2e ms_per_step: the stack in and the result out "
                    "copied at once on two streams, no compute"}


# ----------------------------------------------------------- CPU reference --

class _quiet_stdout:
    """The reference C prints one line per tile whose solver returns non-zero
    (ncs.c:116-119), which a capped run does for most tiles; keep it off the
    JSON stdout."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *a):
        try:
            ctypes.CDLL(None).fflush(None)
        except Exception:
            pass
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def cpu_reduce_frames(frames, gamma, mask_shifted, alpha, max_iters, threads):
    """pyCNCS cReduceNoise on each frame, frames spread over `threads` host
    threads (ctypes releases the GIL).  Returns (wall seconds, kind)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import pycncs
    pycncs.set_overrides(max_iterations=max_iters)
    kind = pycncs.kind()
    g64 = numpy.ascontiguousarray(gamma, dtype=numpy.float64)
    m64 = numpy.ascontiguousarray(mask_shifted, dtype=numpy.float64)
    try:
        with _quiet_stdout():
            t0 = time.perf_counter()
            with ThreadPoolExecutor(max_workers=threads) as ex:
                list(ex.map(lambda fr: pycncs.cReduceNoise(fr, g64, m64, alpha), frames))
            wall = time.perf_counter() - t0
    finally:
        pycncs.set_overrides()
    return wall, kind


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_sample_frames(images_cpu, threads, budget_s=20.0):
    """Frames for a bounded CPU sample: one per thread, at most enough for
    ~budget_s of CPU work and never more than the stack."""
    return min(images_cpu.shape[0], max(1, threads))


def accuracy_gate(w, tile_cost, n_sample, seed=0, tile_u=None, out=None):
    """Per-tile final cost vs the FP64 Newton optimum (oracle) on a random
    sample of tiles: fraction within 1e-4 relative, max and median gap.
    tile_cost: the solver's own per-tile FP64 costs; or tile_u, the final
    tiles [N, 16, 16], whose costs are then computed here in FP64.  With
    ``out`` (the stitched result [T, H, W]) the sampled tiles' owned pixels
    of it -- the interior pixels each tile writes last -- are also compared
    with the optimum, relative to max(|u*|, 1)."""
    from oracle import numpy_ref as nr
    images = w["images"]
    T, H, W = images.shape
    ox, oy = nr.tile_origins(H), nr.tile_origins(W)
    per = len(ox) * len(oy)
    rng = numpy.random.default_rng(seed)
    idx = numpy.sort(rng.choice(T * per, size=min(n_sample, T * per), replace=False))
    gam = numpy.pad(w["gamma"].cpu().numpy().astype(numpy.float64), 1, "edge")
    data, gms = [], []
    cache = {}
    for t in idx:
        f, rem = divmod(int(t), per)
        i, j = divmod(rem, len(oy))
        if f not in cache:
            cache = {f: numpy.pad(images[f].cpu().numpy().astype(numpy.float64), 1, "edge")}
        p = cache[f]
        data.append(p[ox[i]:ox[i] + 16, oy[j]:oy[j] + 16])
        gms.append(gam[ox[i]:ox[i] + 16, oy[j]:oy[j] + 16])
    ms = numpy.fft.fftshift(w["mask"]).astype(numpy.float32).astype(numpy.float64)
    ustar, fstar, _ = nr.newton_solve(numpy.array(data), numpy.array(gms), ms, w["alpha"])
    if tile_cost is None:
        tile_cost = numpy.zeros(T * per)
        tile_cost[idx] = nr.cost(tile_u[idx].astype(numpy.float64), numpy.array(data),
                                 numpy.array(gms), ms, w["alpha"])
    gap = nr.rel_cost_gap(tile_cost[idx], fstar)
    rec = {"tiles_checked": int(idx.size), "frac_within_1e-4": float((gap <= 1e-4).mean()),
           "max_rel_gap": float(gap.max()), "median_rel_gap": float(numpy.median(gap)),
           "referee": "FP64 damped Newton (oracle/numpy_ref.py)"}
    if out is not None:
        own_x = numpy.array([nr.owner_origin(y, ox) for y in range(H)])
        own_y = numpy.array([nr.owner_origin(y, oy) for y in range(W)])
        rel = []
        frames = {}
        for k, t in enumerate(idx):
            f, rem = divmod(int(t), per)
            i, j = divmod(rem, len(oy))
            rows = numpy.nonzero(own_x == ox[i])[0]
            cols = numpy.nonzero(own_y == oy[j])[0]
            if f not in frames:
                frames = {f: out[f].cpu().numpy().astype(numpy.float64)}
            got = frames[f][numpy.ix_(rows, cols)]
            ref = ustar[k][numpy.ix_(rows - ox[i] + 1, cols - oy[j] + 1)]
            rel.append((numpy.abs(got - ref) / numpy.maximum(numpy.abs(ref), 1.0)).ravel())
        rel = numpy.concatenate(rel)
        rec["pixels"] = {"checked": int(rel.size), "max_rel": float(rel.max()),
                         "median_rel": float(numpy.median(rel)),
                         "frac_within_1e-3": float((rel <= 1e-3).mean()),
                         "what": "owned pixels of the sampled tiles in the stitched result "
                                 "vs the FP64 optimum, |u - u*| / max(|u*|, 1)"}
    return rec


def tile_solver_gate(w, solver, n_sample, seed=0, u0_all=None):
    """accuracy_gate for a form whose reported cost is its running value (the
    tensor-core forms): the sampled tiles are solved again through the tile
    entry (which gives the stack path's results exactly) and their exact
    FP64 costs at the returned u are gated."""
    from oracle import numpy_ref as nr
    images = w["images"]
    T, H, W = images.shape
    ox, oy = nr.tile_origins(H), nr.tile_origins(W)
    per = len(ox) * len(oy)
    rng = numpy.random.default_rng(seed)
    idx = numpy.sort(rng.choice(T * per, size=min(n_sample, T * per), replace=False))
    gam = numpy.pad(w["gamma"].cpu().numpy(), 1, "edge")
    data, gms = [], []
    for t in idx:
        f, rem = divmod(int(t), per)
        i, j = divmod(rem, len(oy))
        p = numpy.pad(images[f].cpu().numpy(), 1, "edge")
        data.append(p[ox[i]:ox[i] + 16, oy[j]:oy[j] + 16])
        gms.append(gam[ox[i]:ox[i] + 16, oy[j]:oy[j] + 16])
    data = numpy.ascontiguousarray(numpy.array(data, dtype=numpy.float32))
    gms = numpy.ascontiguousarray(numpy.array(gms, dtype=numpy.float32))
    u0 = None
    if u0_all is not None:
        u0 = u0_all[torch.from_numpy(idx).to(u0_all.device)].contiguous()
    u, _, _, _ = solver.solve_tiles(torch.from_numpy(data).to(images.device),
                                    torch.from_numpy(gms).to(images.device), u0=u0)
    ms = numpy.fft.fftshift(w["mask"]).astype(numpy.float32).astype(numpy.float64)
    d64, g64 = data.astype(numpy.float64), gms.astype(numpy.float64)
    _, fstar, _ = nr.newton_solve(d64, g64, ms, w["alpha"])
    f = nr.cost(u.cpu().numpy().astype(numpy.float64), d64, g64, ms, w["alpha"])
    gap = nr.rel_cost_gap(f, fstar)
    return {"tiles_checked": int(idx.size), "frac_within_1e-4": float((gap <= 1e-4).mean()),
            "max_rel_gap": float(gap.max()), "median_rel_gap": float(numpy.median(gap)),
            "referee": "FP64 damped Newton (oracle/numpy_ref.py), exact cost at the "
                       "returned tiles"}


def cpu_readings(images_cpu, gamma, mask_shifted, alpha, cap, threads):
    """The reference C path (pyCNCS cReduceNoise) on bounded samples of the
    workload, three ways: at the workload's iteration cap on all host
    threads (one frame per thread), to convergence (max_iterations 0, the
    reference's default) on the same frames, and capped on one core (one
    frame).  Returns {reading: {value Mpx/s, cores, sample, seconds}}."""
    T, H, W = images_cpu.shape
    n = cpu_sample_frames(images_cpu, threads)
    frames = [images_cpu[i].astype(numpy.float64) for i in range(n)]
    out = {}
    for name, fr, th, it in (("capped_all_cores", frames, threads, cap),
                             ("unlimited_all_cores", frames, threads, 0),
                             ("capped_one_core", frames[:1], 1, cap)):
        wall, kind = cpu_reduce_frames(fr, gamma, mask_shifted, alpha, it, th)
        out[name] = {"value": len(fr) * H * W / wall / 1e6, "unit": "Mpixel/s", "cores": th,
                     "kind": kind, "seconds": wall,
                     "sample": "%d of %d frames (%dx%d), one per thread, max_iterations=%s"
                               % (len(fr), T, H, W, it if it else "0 (until convergence)")}
    return out


# --------------------------------------------------------------- arms -------

def run_reference(args, world, rank):
    """The reference arm: pyCNCS cReduceNoise (the reference's C path) on the
    host cores, on bounded samples of the workload.  The workload is drawn
    with torch alone (on the GPU when there is one), so this process never
    loads this library's CUDA code."""
    if rank != 0:
        return 0
    from ncs_b200 import sim
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    w = sim.make_stack(args.workload, T=args.frames, device=dev, seed=1234)
    threads = cpu_threads()
    n = cpu_sample_frames(w["images"], threads)
    imgs = w["images"][:n].cpu().numpy()
    T = w["images"].shape[0]
    gamma = w["gamma"].cpu().numpy()
    frames = [imgs[i].astype(numpy.float64) for i in range(n)]
    ms = numpy.fft.fftshift(w["mask"])
    for _ in range(args.warmup):
        cpu_reduce_frames(frames, gamma, ms, w["alpha"], w["max_iters"], threads)
    walls = []
    kind = None
    for _ in range(args.steps):
        wall, kind = cpu_reduce_frames(frames, gamma, ms, w["alpha"], w["max_iters"], threads)
        walls.append(wall)
    H, W = imgs.shape[1:]
    value = n * H * W / (sum(walls) / len(walls)) / 1e6
    sample = ("%d of %d frames (%dx%d) per step, one frame per thread, pyCNCS cReduceNoise "
              "FP64 with libLBFGS-API max_iterations=%d" % (n, T, H, W, w["max_iters"]))
    readings = cpu_readings(imgs, gamma, ms, w["alpha"], w["max_iters"], threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mpixel/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(walls) / len(walls), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(w, args),
        "cpu_baseline": {"value": value, "unit": "Mpixel/s", "cores": threads, "kind": kind,
                         "sample": sample, "readings": readings},
        "e2e": {"value": value, "unit": "Mpixel/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    ref_gpu = reference_gpu(w, args)
    if ref_gpu is not None:
        line["reference_gpu"] = ref_gpu
    print(json.dumps(line), flush=True)
    return 0


def reference_gpu(w, args):
    """The reference's own GPU path on the arm's workload: ncsReduceNoise of
    cuda/ncs.cu compiled unmodified for sm_100a (oracle/_ref), launched as
    cuda/pyCUDANCS/ncs.py launches it, one 16-thread block per tile.  The
    tiles are cut and stitched on the device outside the timed region
    (pyCUDANCS does both on the host); the kernel alone is timed with CUDA
    events.  It runs to its own stopping rule (||g|| <= 1e-4 max(||u||, 1),
    200 iterations at most): the kernel has no cap parameter.  None when the
    kernel was not built or there is no GPU."""
    from oracle import refgpu
    if args.no_compare_plain or not torch.cuda.is_available() or not refgpu.available():
        return None
    dev = torch.device("cuda", 0)
    images, gamma = w["images"].to(dev), w["gamma"].to(dev)
    T, H, W = images.shape
    dt, gt = refgpu.segment(images, gamma)
    ms = numpy.fft.fftshift(w["mask"]).astype(numpy.float32)
    u, it, st = refgpu.reduce_noise_tiles(dt, gt, ms, w["alpha"])   # warm-up
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    reps = max(1, min(args.steps, 2))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        u, it, st = refgpu.reduce_noise_tiles(dt, gt, ms, w["alpha"])
    e1.record(stream)
    torch.cuda.synchronize()
    ms_step = e0.elapsed_time(e1) / reps
    status = {str(k): int(v) for k, v in zip(*numpy.unique(st.cpu().numpy(), return_counts=True))}
    rec = {"kernel": "ncsReduceNoise (cuda/ncs.cu, unmodified, nvcc sm_100a; block 16, grid = "
                     "tiles, as cuda/pyCUDANCS/ncs.py:116-125)",
           "ms_per_step": ms_step, "value": T * H * W / (ms_step / 1e3) / 1e6,
           "unit": "Mpixel/s", "tiles": int(dt.shape[0]),
           "mean_iters": it.double().mean().item(), "status": status,
           "stopping_rule": "||g|| <= 1e-4 max(||u||, 1) or 200 iterations (ncs.cu:55-57)",
           "timed": "kernel only, CUDA events, mean of %d launches after one warm-up" % reps}
    from oracle import numpy_ref as nr
    if dt.shape[0] == T * len(nr.tile_origins(H)) * len(nr.tile_origins(W)):
        rec["accuracy"] = accuracy_gate(w, None, args.accuracy_tiles,
                                        tile_u=u.cpu().numpy())
    del dt, gt, u
    return rec


METRIC = "Mpixel/s at <=1e-4 rel cost vs FP64: warm-start+TC vs plain GPU (pyCNCS ref)"


def workload_config(w, args):
    T, H, W = w["images"].shape
    return {"workload": "%s: %d frames x %dx%d float32, %d WLC chains, alpha %.2f, 16x16 tiles, "
                        "L-BFGS cap %d" % (w["name"], T, H, W, w["cfg"]["chains"], w["alpha"],
                                           w["max_iters"]),
            "frames": T, "height": H, "width": W, "alpha": w["alpha"],
            "max_iters": w["max_iters"], "seed": w["seed"], "form": args.form,
            "ctas_per_sm": args.ctas_per_sm or "library default",
            "l2": "inputs+outputs %.0f MB > 126 MB L2, no flush" % (2 * T * H * W * 4 / 1e6),
            "parallelism": "replicas by frame (one stack per rank)"}


def run_ours(args, world, rank, local):
    import ncs_b200
    from ncs_b200 import sim
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = sim.make_stack(args.workload, T=args.frames, device=dev, seed=1234 + rank)
    images, gamma = w["images"], w["gamma"]
    T, H, W = images.shape
    solver = ncs_b200.Solver(alpha=w["alpha"], max_iters=w["max_iters"], mode=args.form,
                             ctas_per_sm=args.ctas_per_sm)
    solver.set_otf_mask(w["mask"])
    out = torch.empty_like(images)
    stream = torch.cuda.current_stream(dev)

    # untimed statistics run: per-tile iterations / evaluations / final cost
    _, iters, status, cost, evals = solver.reduce_noise(images, gamma, out=out, tile_stats="all")
    torch.cuda.synchronize()
    # the timed launches must reproduce this launch's result bit for bit, so
    # that its per-tile costs are the costs of the timed output
    stats_out = out.clone()
    iters_n = iters.double().sum().item()
    evals_n = evals.double().sum().item()
    n_tiles = iters.numel()
    m = solver.params.m
    # pairs stored when iteration i starts: min(i, m) for i = 0 .. iters-1
    it = iters.double()
    mm = float(m)
    pairs = torch.where(it <= mm, it * (it - 1.0) / 2.0, mm * (mm - 1.0) / 2.0 + (it - mm) * mm)
    flops = (n_tiles * FLOP_INIT + iters_n * FLOP_ITER_BASE[args.form]
             + FLOP_PER_PAIR[args.form] * pairs.sum().item()
             + FLOP_TRIAL * (evals_n - n_tiles))
    st = status.cpu().numpy()

    for _ in range(args.warmup):
        solver.reduce_noise(images, gamma, out=out)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    clocks.begin()
    ev[0].record(stream)
    for k in range(args.steps):
        solver.reduce_noise(images, gamma, out=out)
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    clocks.end()
    barrier(world)
    clk = clocks.stop()
    timed_equal = bool(torch.equal(out, stats_out))
    assert timed_equal, "the timed launches differ from the statistics launch"
    del stats_out
    per_step = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])
    total_ms = max_over_ranks(total_ms, world)
    px = sum_over_ranks(float(T * H * W), world)
    value = px * args.steps / (total_ms / 1e3) / 1e6

    # end to end through the public API from pinned host memory
    h_in = images.cpu().pin_memory()
    h_gamma = gamma.cpu().pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    # at least ~20 stacks: the host link is shared with the machine's other
    # GPUs, so a short window is noisy
    e2e_steps = max(1, min(2 * args.steps, 20))
    solver.reduce_noise_host(h_in, h_gamma, out=h_out)  # warm-up: streams, handles, buffers
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        # every step copies the stack in, solves it and copies it out; the
        # call returns after its last copy completes
        solver.reduce_noise_host(h_in, h_gamma, out=h_out)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
    e2e_value = px * e2e_steps / (e2e_ms / 1e3) / 1e6
    assert torch.equal(h_out, out.cpu()), "e2e result differs from the device-resident run"
    link = host_link_ceiling(h_in, h_out, out, stream)
    link["frac"] = link["both_ms"] / (e2e_ms / e2e_steps)

    # the plain GPU forms (the reference's L-BFGS: scalar initial matrix,
    # Armijo backtracking) on the same stack, for the "vs plain GPU" part of
    # the metric: one warp group per tile (the reference kernel's layout) and
    # one warp per tile (the faster plain kernel)
    plain = {}
    if not args.no_compare_plain and args.form == "spectral":
        for pform in ("plain_wg", "plain"):
            ps = ncs_b200.Solver(alpha=w["alpha"], max_iters=w["max_iters"], mode=pform, m=4)
            ps.set_otf_mask(w["mask"])
            _, p_it, p_st, p_cost = ps.reduce_noise(images, gamma, out=out, tile_stats=True)
            ps.reduce_noise(images, gamma, out=out)
            barrier(world)
            torch.cuda.synchronize()
            pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            nps = max(1, min(args.steps, 3))
            pe0.record(stream)
            for _ in range(nps):
                ps.reduce_noise(images, gamma, out=out)
            pe1.record(stream)
            torch.cuda.synchronize()
            p_ms = max_over_ranks(pe0.elapsed_time(pe1), world) / nps
            plain[pform] = {"form": "%s (m=4)" % pform, "kernel": KERNEL[pform],
                            "ms_per_step": p_ms,
                            "value": px / (p_ms / 1e3) / 1e6,
                            "mean_iters": p_it.double().mean().item(),
                            "capped_tiles": int((p_st == -2).sum().item()),
                            "speedup_of_form": p_ms / (total_ms / args.steps),
                            "_cost": p_cost.cpu().numpy()}
            ps.close()

    # the tensor-core forms on the same stack: the spectral algorithm with the
    # noise term's transforms as tcgen05 GEMMs (TF32; three-way BF16 split)
    tcforms = {}
    pk0 = peaks()[0]
    bf16_peak = pk0.get("bf16_tflops", 1590.0)
    if not args.no_compare_plain and args.form == "spectral":
        for tform in ("tc_tf32", "tc_bf16x3"):
            ts_ = ncs_b200.Solver(alpha=w["alpha"], max_iters=w["max_iters"], mode=tform)
            ts_.set_otf_mask(w["mask"])
            _, t_it, t_st = ts_.reduce_noise(images, gamma, out=out, tile_stats="status")
            ts_.reduce_noise(images, gamma, out=out)
            barrier(world)
            torch.cuda.synchronize()
            te0, te1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ntc = max(1, min(args.steps, 5))
            te0.record(stream)
            for _ in range(ntc):
                ts_.reduce_noise(images, gamma, out=out)
            te1.record(stream)
            torch.cuda.synchronize()
            t_ms = max_over_ranks(te0.elapsed_time(te1), world) / ntc
            passes = t_it.double().sum().item() + n_tiles
            exec_tflops = passes * TC_EXEC_FLOP_PER_PASS[tform] / (t_ms / 1e3) / 1e12
            peak_t = bf16_peak if tform == "tc_bf16x3" else 0.5 * bf16_peak
            st_t = t_st.cpu().numpy()
            tcforms[tform] = {
                "form": "%s (spectral algorithm, m=1)" % tform, "kernel": KERNEL[tform],
                "ms_per_step": t_ms, "value": px / (t_ms / 1e3) / 1e6,
                "mean_iters": t_it.double().mean().item(),
                "status": {str(k): int((st_t == k).sum()) for k in range(-5, 1)
                           if (st_t == k).any()},
                "vs_spectral_fft": (total_ms / args.steps) / t_ms,
                "roofline": {"bound": "tensor", "achieved": exec_tflops, "peak": peak_t,
                             "unit": "TFLOP/s", "frac": exec_tflops / peak_t,
                             "traffic": None, "kernel": KERNEL[tform],
                             "executed_flop_per_pass": TC_EXEC_FLOP_PER_PASS[tform],
                             "dense_q_flop_per_pass": DENSE_Q_FLOP_PER_PASS,
                             "dense_q_equiv_tflops": passes * DENSE_Q_FLOP_PER_PASS
                             / (t_ms / 1e3) / 1e12,
                             "peak_source": "dense BF16, measured burst%s"
                                            % ("" if tform == "tc_bf16x3"
                                               else " x 1/2 (TF32 runs at half the BF16 rate)"),
                             "note": "executed MMA FLOPs over the whole launch; the kernel "
                                     "waits on its four MMA round trips per pass, so the "
                                     "tensor pipe is far from its bound"},
                "_solver": ts_}

    # learned warm start: network inference on the stack, then the spectral
    # solve from its proposals (fallback to the photon image per tile)
    warm = None
    from ncs_b200 import warmstart
    if not args.no_warm_start and args.form == "spectral" and os.path.exists(
            warmstart.DEFAULT_WEIGHTS):
        net = warmstart.WarmStartNet.load()
        # FP32 SIMT inference, for reference
        u0 = net.propose_stack(images, gamma)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        net.propose_stack(images, gamma, out=u0)
        f1.record(stream)
        torch.cuda.synchronize()
        fp32_ms = f0.elapsed_time(f1)
        fp8 = args.warm_precision == "fp8"
        nws = max(1, min(args.steps, 3))
        # tensor-core inference alone in both operand formats
        infer_ms = {}
        for prec in ("bf16", "fp8"):
            net.propose_stack_tc(images, gamma, out=u0, fp8=prec == "fp8")
            torch.cuda.synchronize()
            f0.record(stream)
            for _ in range(nws):
                net.propose_stack_tc(images, gamma, out=u0, fp8=prec == "fp8")
            f1.record(stream)
            torch.cuda.synchronize()
            infer_ms[prec] = f0.elapsed_time(f1) / nws
        # tensor-core inference + solve: the timed leg
        u0, tc_status = net.propose_stack_tc(images, gamma, out=u0, fp8=fp8)
        _, w_it, w_st, w_cost, w_ev, w_fb = solver.reduce_noise_from(images, gamma, u0, out=out)
        barrier(world)
        torch.cuda.synchronize()
        we = [torch.cuda.Event(enable_timing=True) for _ in range(2 * nws + 1)]
        we[0].record(stream)
        for k in range(nws):
            net.propose_stack_tc(images, gamma, out=u0, fp8=fp8)
            we[2 * k + 1].record(stream)
            solver.reduce_noise_from(images, gamma, u0, out=out, stats=False)
            we[2 * k + 2].record(stream)
        torch.cuda.synchronize()
        assert int(tc_status.item()) == 0, "tensor-core inference timed out"
        inf_ms = sum(we[2 * k].elapsed_time(we[2 * k + 1]) for k in range(nws)) / nws
        sol_ms = sum(we[2 * k + 1].elapsed_time(we[2 * k + 2]) for k in range(nws)) / nws
        tot_ms = max_over_ranks(we[0].elapsed_time(we[-1]), world) / nws
        inf_flops = n_tiles * INFER_FLOP_PER_TILE
        pk_tensor = peaks()[0].get("bf16_tflops", 1590.0)  # dense BF16, measured burst
        warm = {"network": "4 x conv3x3 2-32-32-32-1, ReLU, %d params (%s on the tensor "
                           "cores)" % (warmstart.N_PARAMS, "E4M3" if fp8 else "BF16"),
                "kernels": "ncsb::nettc::infer_tc<%s> (tcgen05, %s -> FP32 in TMEM), "
                           "ncs_spectral_kernel<.., Warm>"
                           % (("F8", "kind::f8f6f4 E4M3 x E4M3") if fp8
                              else ("BF16", "kind::f16 BF16 x BF16")),
                "precision": args.warm_precision,
                "ms_infer_fp32_simt": fp32_ms,
                "ms_infer_tc": infer_ms,
                "ms_per_step": tot_ms, "ms_infer": inf_ms, "ms_solve": sol_ms,
                "value": px / (tot_ms / 1e3) / 1e6,
                "mean_iters": w_it.double().mean().item(),
                "mean_iters_photon_start": iters_n / n_tiles,
                "mean_evals": w_ev.double().mean().item(),
                "fallback_frac": w_fb.double().mean().item(),
                "infer_tflops": inf_flops / (inf_ms / 1e3) / 1e12,
                "infer_tensor_frac": inf_flops / (inf_ms / 1e3) / 1e12
                / (pk_tensor * (2.0 if fp8 else 1.0)),
                "infer_tensor_peak": "dense %s, measured BF16 burst%s"
                                     % ("E4M3" if fp8 else "BF16", " x 2" if fp8 else ""),
                "infer_flop_per_tile": INFER_FLOP_PER_TILE,
                "speedup_vs_photon_start": (total_ms / args.steps) / tot_ms,
                "_cost": w_cost.cpu().numpy()}
        # the warm start with a tensor-core solve: tensor-core inference, then
        # the TF32 tensor-core form from its proposals
        if "tc_tf32" in tcforms:
            tsv = tcforms["tc_tf32"]["_solver"]
            _, wt_it, wt_st, _, _, wt_fb = tsv.reduce_noise_from(images, gamma, u0, out=out)
            barrier(world)
            torch.cuda.synchronize()
            wt = [torch.cuda.Event(enable_timing=True) for _ in range(2 * nws + 1)]
            wt[0].record(stream)
            for k in range(nws):
                net.propose_stack_tc(images, gamma, out=u0, fp8=fp8)
                wt[2 * k + 1].record(stream)
                tsv.reduce_noise_from(images, gamma, u0, out=out, stats=False)
                wt[2 * k + 2].record(stream)
            torch.cuda.synchronize()
            wt_tot = max_over_ranks(wt[0].elapsed_time(wt[-1]), world) / nws
            wt_sol = sum(wt[2 * k + 1].elapsed_time(wt[2 * k + 2]) for k in range(nws)) / nws
            st_w = wt_st.cpu().numpy()
            warm["tc_form"] = {
                "kernels": "ncsb::nettc::infer_tc<%s>, ncs_tc_kernel<TF32, Warm>"
                           % ("F8" if fp8 else "BF16"),
                "ms_per_step": wt_tot, "ms_solve": wt_sol,
                "value": px / (wt_tot / 1e3) / 1e6,
                "mean_iters": wt_it.double().mean().item(),
                "fallback_frac": wt_fb.double().mean().item(),
                "status": {str(k): int((st_w == k).sum()) for k in range(-5, 1)
                           if (st_w == k).any()},
                "_u0": u0.clone()}
        del u0

    pk, pk_src = peaks()
    n_sms = torch.cuda.get_device_properties(dev).multi_processor_count
    fp32_peak = fp32_peak_tflops(pk.get("sm_max_mhz", 1965.0), n_sms)
    launch_ms = statistics.mean(per_step)
    wipp = WARP_INST_PER_PASS.get(args.form)
    inst_launch = wipp * (iters_n + n_tiles) if wipp else None
    issue_peak = n_sms * 4 * pk.get("sm_max_mhz", 1965.0) * 1e6
    achieved = flops / (launch_ms / 1e3) / 1e12
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            tj = json.load(f)
        key = "%s/%s" % (args.workload, args.form)
        if key in tj:
            traffic = tj[key]["bytes_per_launch"]
    alg_bytes = 8.0 * T * H * W + 4.0 * H * W
    line = {
        "metric": METRIC, "value": value, "unit": "Mpixel/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded WLC structure + sCMOS camera model)",
        "config": workload_config(w, args),
        "frames_per_s": world * T * args.steps / (total_ms / 1e3),
        "tiles": n_tiles, "mean_iters": iters_n / n_tiles, "mean_evals": evals_n / n_tiles,
        "status": {str(k): int((st == k).sum()) for k in range(-5, 1) if (st == k).any()},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                     "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": traffic,
                     "kernel": KERNEL[args.form],
                     "peak_source": "148 SMs x 128 FP32 lanes x 2 x %s sm_max_mhz (%s)"
                                    % (pk.get("sm_max_mhz"), pk_src),
                     "flops_per_launch": flops,
                     "hbm": {"algorithmic_bytes": alg_bytes,
                             "achieved_gbs": alg_bytes / (launch_ms / 1e3) / 1e9,
                             "peak_gbs": pk.get("hbm_gbs")},
                     "issue": None if not wipp else {"est_warp_inst_per_launch": inst_launch,
                               "achieved_warp_inst_per_s": inst_launch / (launch_ms / 1e3),
                               "peak_warp_inst_per_s": issue_peak,
                               "frac": inst_launch / (launch_ms / 1e3) / issue_peak,
                               "source": "warp instructions per pass from one ncu capture "
                                         "of the kernel on stack512 at 64 frames (commit %s) "
                                         "x passes counted in this run; peak = SMs x 4 "
                                         "schedulers x sm_max_mhz"
                                         % WARP_INST_MEASURED.get(args.form)}},
        "e2e": {"value": e2e_value, "unit": "Mpixel/s",
                "h2d_bytes_per_step": int(h_in.numel() * 4 + h_gamma.numel() * 4),
                "d2h_bytes_per_step": int(h_out.numel() * 4),
                "api": "ncs_b200.Solver.reduce_noise_host -> ncsb_reduce_noise_host: pinned "
                       "host buffers; T/40-frame chunks round-robin over 4 streams, each copying "
                       "in, solving and copying out",
                "ms_per_step": e2e_ms / e2e_steps,
                "roofline": link},
        "gpu_launches": args.steps,
        "clocks": clk,
    }
    for pform, rec in plain.items():
        line["plain_gpu" if pform == "plain_wg" else "plain_gpu_warp"] = {
            k: v for k, v in rec.items() if not k.startswith("_")}
    if tcforms:
        line["tensor_core_forms"] = {f_: {k: v for k, v in rec.items() if not k.startswith("_")}
                                     for f_, rec in tcforms.items()}
    if warm is not None:
        line["warm_start"] = {k: v for k, v in warm.items() if not k.startswith("_")}
        if "tc_form" in warm:
            line["warm_start"]["tc_form"] = {k: v for k, v in warm["tc_form"].items()
                                             if not k.startswith("_")}
    if warm is not None and "plain_wg" in plain:
        # the metric's named comparison: the warm-start + tensor-core form
        # against the plain GPU kernel (one warp group per tile), and the same
        # ratio for the other forms on this stack
        line["metric_form"] = {
            "warm_tc_over_plain_gpu": warm["value"] / plain["plain_wg"]["value"],
            "warm_tc_over_plain_gpu_warp": warm["value"] / plain["plain"]["value"],
            "spectral_over_plain_gpu": value / plain["plain_wg"]["value"],
            "target": ">= 3x the plain GPU kernel at equal accuracy"}
        if "tc_form" in warm:
            line["metric_form"]["warm_tc_form_over_plain_gpu"] = (
                warm["tc_form"]["value"] / plain["plain_wg"]["value"])
        for f_, rec in tcforms.items():
            line["metric_form"]["%s_over_plain_gpu" % f_] = (
                rec["value"] / plain["plain_wg"]["value"])
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = cpu_threads()
        n = cpu_sample_frames(images, threads)
        readings = cpu_readings(images[:n].cpu().numpy(), gamma.cpu().numpy(),
                                numpy.fft.fftshift(w["mask"]), w["alpha"], w["max_iters"],
                                threads)
        cap = readings["capped_all_cores"]
        line["cpu_baseline"] = {
            "value": cap["value"], "unit": "Mpixel/s", "cores": threads, "kind": cap["kind"],
            "sample": "%d of %d frames, one per thread, pyCNCS cReduceNoise FP64, "
                      "max_iterations=%d" % (n, T, w["max_iters"]),
            "readings": readings}
        line["accuracy"] = accuracy_gate(w, cost.cpu().numpy(), args.accuracy_tiles, out=out)
        line["accuracy"]["timed_output"] = ("bit-identical to the statistics launch whose "
                                            "per-tile costs are gated: %s" % timed_equal)
        for pform, rec in plain.items():
            key = "plain_gpu" if pform == "plain_wg" else "plain_gpu_warp"
            line[key]["accuracy"] = accuracy_gate(w, rec["_cost"], args.accuracy_tiles)
        if warm is not None:
            line["warm_start"]["accuracy"] = accuracy_gate(w, warm["_cost"], args.accuracy_tiles)
        for f_, rec in tcforms.items():
            line["tensor_core_forms"][f_]["accuracy"] = tile_solver_gate(
                w, rec["_solver"], args.accuracy_tiles)
        if warm is not None and "tc_form" in warm:
            line["warm_start"]["tc_form"]["accuracy"] = tile_solver_gate(
                w, tcforms["tc_tf32"]["_solver"], args.accuracy_tiles,
                u0_all=warm["tc_form"]["_u0"])
    for rec in tcforms.values():
        rec["_solver"].close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def mixed_accuracy(stacks, cost, n_sample, seed=0):
    """accuracy_gate over a batch: a random sample of tiles across all stacks,
    each checked against the FP64 optimum with its own stack's alpha and mask."""
    from oracle import numpy_ref as nr
    per, offs = [], [0]
    for st in stacks:
        T, H, W = st["images"].shape
        per.append(len(nr.tile_origins(H)) * len(nr.tile_origins(W)))
        offs.append(offs[-1] + T * per[-1])
    rng = numpy.random.default_rng(seed)
    idx = numpy.sort(rng.choice(offs[-1], size=min(n_sample, offs[-1]), replace=False))
    gaps = []
    for t in idx:
        k = int(numpy.searchsorted(offs, t, side="right") - 1)
        st = stacks[k]
        f, rem = divmod(int(t - offs[k]), per[k])
        H, W = st["images"].shape[1:]
        ox, oy = nr.tile_origins(H), nr.tile_origins(W)
        i, j = divmod(rem, len(oy))
        im = numpy.pad(st["images"][f].cpu().numpy().astype(numpy.float64), 1, "edge")
        g = st["gamma"].cpu().numpy().astype(numpy.float64)
        g = numpy.pad(g if g.ndim == 2 else g[f], 1, "edge")
        ms = numpy.fft.fftshift(st["mask"]).astype(numpy.float32).astype(numpy.float64)
        _, fstar, _ = nr.newton_solve(im[None, ox[i]:ox[i] + 16, oy[j]:oy[j] + 16],
                                      g[None, ox[i]:ox[i] + 16, oy[j]:oy[j] + 16], ms,
                                      st["alpha"])
        gaps.append(float(nr.rel_cost_gap(cost[t:t + 1], fstar)[0]))
    gaps = numpy.array(gaps)
    return {"tiles_checked": int(idx.size), "frac_within_1e-4": float((gaps <= 1e-4).mean()),
            "max_rel_gap": float(gaps.max()), "median_rel_gap": float(numpy.median(gaps)),
            "referee": "FP64 damped Newton (oracle/numpy_ref.py), per stack alpha and mask"}


def run_mixed(args, world, rank, local):
    """The mixed-workload batch: 64 stacks (own shape, alpha, mask) solved by
    one batched launch captured in a CUDA graph, launch parameters chosen by
    the autotuner.  One batch per rank (replicas)."""
    import ncs_b200
    from ncs_b200 import sim, tune
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stacks = sim.make_mixed(args.stacks, seed=4242 + rank, device=dev)
    px = float(sum(st["images"].numel() for st in stacks))
    solver = ncs_b200.Solver(max_iters=200)
    outs = solver.batch_set(stacks)
    stats = solver.batch_stats()
    best, tried = tune.autotune(solver, lambda: solver.batch_reduce_noise(), tune.batch_key(solver))
    solver.batch_reduce_noise(stats=stats)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        solver.batch_reduce_noise()
    for _ in range(args.warmup):
        graph.replay()
    stream = torch.cuda.current_stream(dev)
    clocks = Clocks(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.begin()
    e0.record(stream)
    for _ in range(args.steps):
        graph.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks.end()
    barrier(world)
    clk = clocks.stop()
    total_ms = max_over_ranks(e0.elapsed_time(e1), world)
    value = sum_over_ranks(px, world) * args.steps / (total_ms / 1e3) / 1e6

    # end to end: pinned host stacks in, one batched solve, results out (only
    # when the host can pin both copies of the batch with room to spare)
    import psutil
    e2e = None
    need = 2 * 4 * px
    if psutil.virtual_memory().available > 3 * need:
        h_in = [st["images"].cpu().pin_memory() for st in stacks]
        h_out = [torch.empty_like(h).pin_memory() for h in h_in]
        e2e_steps = max(1, min(args.steps, 3))
        barrier(world)
        torch.cuda.synchronize()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for _ in range(e2e_steps):
            for st, h in zip(stacks, h_in):
                st["images"].copy_(h, non_blocking=True)
            graph.replay()
            for o, h in zip(outs, h_out):
                h.copy_(o, non_blocking=True)
        e3.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(e2.elapsed_time(e3), world)
        e2e = {"value": sum_over_ranks(px, world) * e2e_steps / (e2e_ms / 1e3) / 1e6,
               "unit": "Mpixel/s",
               "h2d_bytes_per_step": int(sum(h.numel() * 4 for h in h_in)),
               "d2h_bytes_per_step": int(sum(h.numel() * 4 for h in h_out)),
               "api": "per-stack pinned copies + Solver.batch_reduce_noise (graph replay), "
                      "one stream"}
        del h_in, h_out
    else:
        e2e = {"value": None, "unit": "Mpixel/s", "h2d_bytes_per_step": 0,
               "d2h_bytes_per_step": 0,
               "skipped": "host RAM below 3x the %.1f GB of pinned copies" % (need / 1e9)}
    # learned warm start over the batch: tensor-core inference, then the batched
    # solve from its proposals, both kernels captured in one CUDA graph
    warm = None
    from ncs_b200 import warmstart
    if not args.no_warm_start and os.path.exists(warmstart.DEFAULT_WEIGHTS):
        net = warmstart.WarmStartNet.load(device=dev)
        fp8 = args.warm_precision == "fp8"
        u0 = torch.empty((solver.batch_tiles, 16, 16), dtype=torch.float32, device=dev)
        tc_status = torch.zeros(1, dtype=torch.int32, device=dev)
        w_stats = solver.batch_stats()
        net.propose_batch_tc(solver, out=u0, status=tc_status, fp8=fp8)
        solver.batch_reduce_noise(u0_tiles=u0, stats=w_stats)
        torch.cuda.synchronize()
        wgraph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(wgraph):
            net.propose_batch_tc(solver, out=u0, status=tc_status, fp8=fp8)
            solver.batch_reduce_noise(u0_tiles=u0)
        for _ in range(args.warmup):
            wgraph.replay()
        barrier(world)
        torch.cuda.synchronize()
        nws = max(1, min(args.steps, 3))
        w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0.record(stream)
        for _ in range(nws):
            wgraph.replay()
        w1.record(stream)
        torch.cuda.synchronize()
        assert int(tc_status.item()) == 0, "tensor-core inference timed out"
        w_ms = max_over_ranks(w0.elapsed_time(w1), world) / nws
        # the inference alone, for the split
        i0, i1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        i0.record(stream)
        net.propose_batch_tc(solver, out=u0, status=tc_status, fp8=fp8)
        i1.record(stream)
        torch.cuda.synchronize()
        warm = {"kernels": "ncsb::nettc::infer_tc<%s> over the batch's stack descriptors, "
                           "then ncs_spectral_kernel<.., Warm, Batch>, one CUDA graph"
                           % ("F8" if fp8 else "BF16"),
                "precision": args.warm_precision,
                "ms_per_step": w_ms, "ms_infer": i0.elapsed_time(i1),
                "value": sum_over_ranks(px, world) / (w_ms / 1e3) / 1e6,
                "mean_iters": w_stats["iters"].double().mean().item(),
                "fallback_frac": w_stats["start"].double().mean().item(),
                "speedup_vs_photon_start": (total_ms / args.steps) / w_ms,
                "_cost": w_stats["cost"].cpu().numpy()}
        # the same with the TF32 tensor-core form solving the batch from the
        # proposals (the mixed workload's warm start + tensor-core noise term)
        tsolver = ncs_b200.Solver(max_iters=200, mode="tc_tf32")
        touts = tsolver.batch_set(stacks)
        t_stats = tsolver.batch_stats()
        net.propose_batch_tc(tsolver, out=u0, status=tc_status, fp8=fp8)
        tsolver.batch_reduce_noise(u0_tiles=u0, stats=t_stats)
        torch.cuda.synchronize()
        tgraph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(tgraph):
            net.propose_batch_tc(tsolver, out=u0, status=tc_status, fp8=fp8)
            tsolver.batch_reduce_noise(u0_tiles=u0)
        for _ in range(args.warmup):
            tgraph.replay()
        barrier(world)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(nws):
            tgraph.replay()
        t1.record(stream)
        torch.cuda.synchronize()
        assert int(tc_status.item()) == 0, "tensor-core inference timed out"
        t_ms = max_over_ranks(t0.elapsed_time(t1), world) / nws
        st_t = t_stats["status"].cpu().numpy()
        warm["tc_form"] = {
            "kernels": "ncsb::nettc::infer_tc<%s>, then ncs_tc_kernel<TF32, Warm, Batch>, "
                       "one CUDA graph" % ("F8" if fp8 else "BF16"),
            "ms_per_step": t_ms, "value": sum_over_ranks(px, world) / (t_ms / 1e3) / 1e6,
            "mean_iters": t_stats["iters"].double().mean().item(),
            "fallback_frac": t_stats["start"].double().mean().item(),
            "status": {str(k): int((st_t == k).sum()) for k in range(-5, 1) if (st_t == k).any()},
            "_cost": t_stats["cost"].cpu().numpy()}
        del tgraph, touts
        tsolver.close()
        del wgraph, u0

    sides = sorted({st["side"] for st in stacks})
    line = {
        "metric": METRIC, "value": value, "unit": "Mpixel/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded chains or beads, sCMOS camera model)",
        "config": {"workload": "mixed%d: %d stacks, sides %s, %d frames in all, own alpha "
                               "U(0.05,0.5) / NA / wavelength / mask per stack, spectral form, "
                               "one batched launch replayed from a CUDA graph"
                               % (len(stacks), len(stacks), sides,
                                  sum(st["T"] for st in stacks)),
                   "pixels": px, "tiles": solver.batch_tiles, "autotuned": best,
                   "parallelism": "replicas (one batch per rank)"},
        "mean_iters": stats["iters"].double().mean().item(),
        "status": {str(k): int((stats["status"] == k).sum()) for k in range(-5, 1)},
        "autotune_ms": tried,
        "e2e": e2e,
        "gpu_launches": args.steps,
        "clocks": clk,
    }
    if warm is not None:
        line["warm_start"] = {k: v for k, v in warm.items() if not k.startswith("_")}
        line["warm_start"]["tc_form"] = {k: v for k, v in warm["tc_form"].items()
                                         if not k.startswith("_")}
    if rank == 0:
        line["accuracy"] = mixed_accuracy(stacks, stats["cost"].cpu().numpy(),
                                          args.accuracy_tiles)
        if warm is not None:
            line["warm_start"]["accuracy"] = mixed_accuracy(stacks, warm["_cost"],
                                                            args.accuracy_tiles)
            # the tensor-core form reports its running cost (v = 2 alpha Q u kept
            # by updates), which differs from the exact cost by its transform error
            line["warm_start"]["tc_form"]["accuracy"] = mixed_accuracy(
                stacks, warm["tc_form"]["_cost"], args.accuracy_tiles)
            line["warm_start"]["tc_form"]["accuracy"]["cost"] = "the kernel's running cost"
        print(json.dumps(line), flush=True)
    del graph
    return 0


def run_adu(args, world, rank, local):
    """Raw camera frames -- 16-bit counts, as an sCMOS camera writes them --
    through the device preprocessing prologue (Solver.reduce_noise_adu: one
    conversion kernel, ADU -> photo-electrons and gamma, then the solve)
    against the two-step path of the reference's scripts written in torch
    (elementwise conversion, then solve), on a stack512-sized stack of
    simulated raw frames.  e2e: host counts in, host photo-electrons out
    through the pipelined Solver.reduce_noise_adu_host.  Replicas by frame."""
    import ncs_b200
    from ncs_b200 import sim
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = sim.make_stack_gpu("stack512", T=args.frames, device=dev, seed=1234 + rank, adu=True)
    adu = w["adu"].round().clamp(0.0, 65535.0).to(torch.uint16)
    off, gain, var = w["offset"], w["gain"], w["var"]
    T, H, W = adu.shape
    solver = ncs_b200.Solver(alpha=w["alpha"], max_iters=w["max_iters"])
    solver.set_otf_mask(w["mask"])
    out = torch.empty(adu.shape, dtype=torch.float32, device=dev)
    gamma = var / (gain * gain)

    def two_step():
        d = (adu.float() - off) / gain
        d = torch.where(d <= 0, torch.full_like(d, 1e-6), d)
        return solver.reduce_noise(d, gamma)

    ours = solver.reduce_noise_adu(adu, off, gain, var, out=out)
    torch.cuda.synchronize()
    exact = bool(torch.equal(ours, two_step()))
    stream = torch.cuda.current_stream(dev)

    def timed(fn, n):
        for _ in range(args.warmup):
            fn()
        barrier(world)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(n):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(a.elapsed_time(b), world)

    clocks = Clocks(local)
    clocks.start()
    clocks.begin()
    total_ms = timed(lambda: solver.reduce_noise_adu(adu, off, gain, var, out=out), args.steps)
    clocks.end()
    clk = clocks.stop()
    two_ms = timed(two_step, args.steps)
    px = sum_over_ranks(float(T * H * W), world)
    value = px * args.steps / (total_ms / 1e3) / 1e6

    # end to end: raw counts from pinned host memory, photo-electrons back,
    # through the pipelined host entry
    h_adu = adu.cpu().pin_memory()
    h_out = torch.empty(adu.shape, dtype=torch.float32).pin_memory()
    steps2 = max(1, min(2 * args.steps, 20))
    e2e_ms = timed(lambda: solver.reduce_noise_adu_host(h_adu, off, gain, var, out=h_out), steps2)
    assert torch.equal(h_out, out.cpu()), "e2e result differs from the device-resident run"
    link = host_link_ceiling(h_adu, h_out, out, stream)
    link["frac"] = link["both_ms"] / (e2e_ms / steps2)
    line = {
        "metric": "Mpixel/s, raw ADU frames through the device preprocessing prologue",
        "value": value, "unit": "Mpixel/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (u16 counts in)",
        "data": "synthetic raw frames (GPU simulator: WLC structure, sCMOS offset/gain/"
                "variance maps, Poisson + read noise, rounded to 16-bit counts)",
        "config": {"workload": "adu: stack512 raw frames (%d x %dx%d uint16 ADU), one "
                               "gain/variance map pair, spectral form" % (T, H, W),
                   "frames": T, "height": H, "width": W,
                   "l2": "inputs+outputs %.0f MB > 126 MB L2, no flush" % (6 * T * H * W / 1e6),
                   "parallelism": "replicas by frame (one stack per rank)"},
        "two_step": {"ms_per_step": two_ms / args.steps,
                     "api": "torch elementwise ADU -> photo-electrons, then Solver.reduce_noise",
                     "result_equal": exact},
        "speedup_vs_two_step": two_ms / total_ms,
        "launches_per_step": "conversion kernel + solver kernel",
        "e2e": {"value": px * steps2 / (e2e_ms / 1e3) / 1e6, "unit": "Mpixel/s",
                "h2d_bytes_per_step": int(h_adu.numel() * h_adu.element_size()),
                "d2h_bytes_per_step": int(h_out.numel() * 4),
                "ms_per_step": e2e_ms / steps2,
                "api": "Solver.reduce_noise_adu_host -> ncsb_reduce_noise_adu_host: pinned "
                       "16-bit counts in, T/40-frame chunks over 4 streams, each copying "
                       "counts in, converting, solving and copying photo-electrons out",
                "roofline": link},
        "gpu_launches": 2 * args.steps,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_normalized(args, world, rank, local):
    """The normalised single-pixel variant (the reference's MATLAB package,
    ncsb_reduce_noise_normalized) on the stack512 stack with its demos'
    settings: alpha 1, 15 iterations, the 3 x 3 genfilter mask of twice the
    NA.  One launch per step (one thread per pixel); replicas by frame."""
    import ncs_b200
    from ncs_b200 import otf, sim
    from oracle import normalized_ref as nref
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = sim.make_stack("stack512", T=args.frames, device=dev, seed=1234 + rank)
    images, gamma = w["images"], w["gamma"]
    T, H, W = images.shape
    mask = otf.normalized_mask(0.1, 1.4, 0.7)
    alpha, cap = 1.0, 15
    out, it, st, cost = ncs_b200.reduce_noise_normalized(images, gamma, mask, alpha=alpha,
                                                         max_iters=cap, stats=True)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        ncs_b200.reduce_noise_normalized(images, gamma, mask, alpha=alpha, max_iters=cap)
    stream = torch.cuda.current_stream(dev)
    clocks = Clocks(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.begin()
    e0.record(stream)
    for _ in range(args.steps):
        ncs_b200.reduce_noise_normalized(images, gamma, mask, alpha=alpha, max_iters=cap)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks.end()
    barrier(world)
    clk = clocks.stop()
    total_ms = max_over_ranks(e0.elapsed_time(e1), world)
    px = sum_over_ranks(float(T * H * W), world)
    value = px * args.steps / (total_ms / 1e3) / 1e6

    # end to end: pinned host stack in, solve, result out, on one stream
    h_in = images.cpu().pin_memory()
    h_g = gamma.cpu().pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    steps2 = max(1, min(args.steps, 5))
    barrier(world)
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(steps2):
        images.copy_(h_in, non_blocking=True)
        gamma.copy_(h_g, non_blocking=True)
        o = ncs_b200.reduce_noise_normalized(images, gamma, mask, alpha=alpha, max_iters=cap)
        h_out.copy_(o, non_blocking=True)
    e3.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e2.elapsed_time(e3), world)

    stv = st.cpu().numpy()
    line = {
        "metric": "Mpixel/s, normalised single-pixel NCS variant (3x3 segment per pixel)",
        "value": value, "unit": "Mpixel/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded WLC structure + sCMOS camera model)",
        "config": {"workload": "normalized: stack512 (%d frames x %dx%d), alpha %.1f, BFGS cap "
                               "%d, 3x3 genfilter mask of 2 NA (the reference demos' settings)"
                               % (T, H, W, alpha, cap),
                   "frames": T, "height": H, "width": W,
                   "l2": "inputs+outputs %.0f MB > 126 MB L2, no flush" % (2 * T * H * W * 4 / 1e6),
                   "parallelism": "replicas by frame (one stack per rank)"},
        "mean_iters": float(it.double().mean().item()),  # per pixel
        "status": {str(k): int((stv == k).sum()) for k in range(-5, 1) if (stv == k).any()},
        "e2e": {"value": px * steps2 / (e2e_ms / 1e3) / 1e6, "unit": "Mpixel/s",
                "h2d_bytes_per_step": int(h_in.numel() * 4 + h_g.numel() * 4),
                "d2h_bytes_per_step": int(h_out.numel() * 4),
                "api": "pinned copies + ncs_b200.reduce_noise_normalized, one stream"},
        "gpu_launches": args.steps,
        "clocks": clk,
    }
    if rank == 0:
        # accuracy: per-pixel final cost vs the FP64 Newton optimum of its segment
        rng = numpy.random.default_rng(0)
        n = T * H * W
        idx = rng.choice(n, size=min(args.accuracy_tiles, n), replace=False)
        im = images.cpu().numpy().astype(numpy.float64)
        gm = gamma.cpu().numpy().astype(numpy.float64)
        cst = cost.cpu().numpy().reshape(-1)
        m64 = numpy.asarray(mask, dtype=numpy.float32).astype(numpy.float64)
        gaps, t0 = [], time.time()
        for k in idx:
            f, rem = divmod(int(k), H * W)
            y, x = divmod(rem, W)
            ys = numpy.clip(numpy.arange(y - 1, y + 2), 0, H - 1)
            xs = numpy.clip(numpy.arange(x - 1, x + 2), 0, W - 1)
            _, fstar = nref.newton(im[f][numpy.ix_(ys, xs)], gm[numpy.ix_(ys, xs)], m64, alpha)
            gaps.append((cst[k] - fstar) / max(abs(fstar), 1.0))
        cpu_s = time.time() - t0
        gaps = numpy.array(gaps)
        line["accuracy"] = {"pixels_checked": int(idx.size),
                            "frac_within_1e-4": float((gaps <= 1e-4).mean()),
                            "max_rel_gap": float(gaps.max()),
                            "median_rel_gap": float(numpy.median(gaps)),
                            "referee": "FP64 damped Newton per segment "
                                       "(oracle/normalized_ref.py), run to convergence"}
        line["cpu_baseline"] = {"value": idx.size / cpu_s / 1e6, "unit": "Mpixel/s", "cores": 1,
                                "kind": "port",
                                "sample": "%d pixels, FP64 Newton per 3x3 segment in numpy (the "
                                          "MATLAB fminunc reference cannot run here)" % idx.size}
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40,
                    help="timed steps (40 x ~2.3 ms gives the clock sampler a few samples)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="sensor2048",
                    help="sensor2048 (default: 100 x 2048^2, 60 chains, 0.5%% hot pixels), "
                         "stack512, frame256, mixed, adu or normalized")
    ap.add_argument("--frames", type=int, default=None, help="override the frame count")
    ap.add_argument("--form", default="spectral", choices=sorted(KERNEL))
    ap.add_argument("--no-compare-plain", action="store_true",
                    help="skip timing the plain form on the same stack")
    ap.add_argument("--warm-precision", choices=["fp8", "bf16"], default="fp8",
                    help="operand format of the warm start's tensor-core inference")
    ap.add_argument("--no-warm-start", action="store_true",
                    help="skip the learned warm-start leg")
    ap.add_argument("--accuracy-tiles", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ctas-per-sm", type=int, default=0,
                    help="resident CTAs per SM of the solve (0: the library's default)")
    ap.add_argument("--stacks", type=int, default=64,
                    help="stacks in the mixed workload (--workload mixed)")
    args = ap.parse_args()
    if args.impl == "reference":
        # rank 0 alone times the CPU path; no process group is needed
        return run_reference(args, int(os.environ.get("WORLD_SIZE", "1")),
                             int(os.environ.get("RANK", "0")))
    world, rank, local = dist_setup()
    try:
        if args.workload == "mixed":
            return run_mixed(args, world, rank, local)
        if args.workload == "normalized":
            return run_normalized(args, world, rank, local)
        if args.workload == "adu":
            return run_adu(args, world, rank, local)
        return run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
