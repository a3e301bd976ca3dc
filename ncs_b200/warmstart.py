"""Learned warm start for the NCS solve.

A 4-layer 3x3 convolutional network (2 -> 32 -> 32 -> 32 -> 1 channels, ReLU
after the first three layers, 19,393 FP32 parameters) maps each 16x16 tile's
photon image d and gamma map to a proposed start u0 for the L-BFGS solve; the
solver (``Solver.reduce_noise_from``) starts each tile at the proposal unless
the proposal's cost is higher than the photon image's, so the unchanged
stopping rule decides convergence and the plain start is the fallback.  The
reference has no learned part: its solves always start at u = d
(clib/pyCNCS/ncs.c:548-551, cuda/ncs.cu:933).

Everything runs on the project's own kernels (libncs_b200.so, ``ncsb_net_*``):
forward convolutions, weight gradients, input gradients through flipped
weights, ReLU backward, the MSE loss gradient, Adam and the fused inference
kernel.  PyTorch only allocates buffers and does index plumbing for the
training data.

Training data: seeded 512 x 512 simulations (rendered and sampled on the GPU,
ncs_b200/sim.py make_stack_gpu) with the full-sensor workload's structure
density and camera (hot pixels included), per-emitter photons U(50, 400) and
background U(2, 30) photons/px, cut into
tiles with the solvers' segmentation and solved to convergence by the plain
GPU kernel (epsilon 1e-6).  The regression target is the normalised
correction y* = (u* - d) / s with s the tile's standard deviation + 1.
"""
import argparse
import ctypes
import math
import os

import numpy
import torch

from . import _lib
from .ncs import Solver, _ptr, launch_stream

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "warmstart_params.npy")

C = 32
# (cin, cout, relu) of the four layers, in the order of the packed vector
LAYERS = ((2, C, True), (C, C, True), (C, C, True), (C, 1, False))


def layer_offsets():
    """[(w_offset, w_size, b_offset, b_size)] of each layer in the packed vector."""
    out, o = [], 0
    for cin, cout, _ in LAYERS:
        nw = cin * 9 * cout
        out.append((o, nw, o + nw, cout))
        o += nw + cout
    return out


N_PARAMS = sum(cin * 9 * cout + cout for cin, cout, _ in LAYERS)


def init_params(seed=0):
    """He-normal weights for the ReLU layers, zero biases, zero last layer
    (the untrained network proposes u0 = d)."""
    rng = numpy.random.default_rng(seed)
    p = numpy.zeros(N_PARAMS, dtype=numpy.float32)
    for (wo, nw, bo, nb), (cin, cout, relu) in zip(layer_offsets(), LAYERS):
        if relu:
            p[wo:wo + nw] = rng.normal(0.0, math.sqrt(2.0 / (cin * 9)), nw)
    return p


def _stream_ptr(stream, device, *tensors):
    """The launch stream as a C pointer (ncs.launch_stream: a caller's stream
    waits for the current one, and ``tensors`` are recorded on it)."""
    return ctypes.c_void_p(launch_stream(stream, device, *tensors).cuda_stream)


class WarmStartNet:
    """The network's parameters on one CUDA device plus its kernels."""

    def __init__(self, params=None, device=None, seed=0):
        self.lib = _lib.load()
        if self.lib.ncsb_net_param_count() != N_PARAMS:
            raise RuntimeError("library and Python disagree on the network size")
        self.device = torch.device(device if device is not None else "cuda")
        if params is None:
            params = init_params(seed)
        p = torch.as_tensor(numpy.asarray(params, dtype=numpy.float32).reshape(-1))
        if p.numel() != N_PARAMS:
            raise ValueError("expected %d parameters, got %d" % (N_PARAMS, p.numel()))
        self.params = p.to(self.device).contiguous()
        self._adam = None
        self._bufs = {}

    # ---- persistence --------------------------------------------------------
    @classmethod
    def load(cls, path=DEFAULT_WEIGHTS, device=None):
        return cls(numpy.load(path), device=device)

    def save(self, path):
        numpy.save(path, self.params.cpu().numpy())

    def _check(self, rc, what):
        if rc != _lib.NCSB_OK:
            raise RuntimeError("%s failed with code %d" % (what, rc))

    def _slices(self, vec):
        out = []
        for wo, nw, bo, nb in layer_offsets():
            out.append((vec[wo:wo + nw], vec[bo:bo + nb]))
        return out

    # ---- inference ----------------------------------------------------------
    def propose_stack(self, images, gamma, out=None, stream=None):
        """Proposals [n_tiles, 16, 16] for a [T, H, W] stack (gamma [H, W] or
        [T, H, W]), tiles in (frame, tile-row, tile-col) order."""
        T, H, W = images.shape
        per_frame = 1 if gamma.dim() == 3 else 0
        n = _lib.num_tiles(T, H, W)
        if out is None:
            out = torch.empty((n, 16, 16), dtype=torch.float32, device=self.device)
        images, gamma = images.contiguous(), gamma.contiguous()
        sp = _stream_ptr(stream, self.device, self.params, images, gamma, out)
        with torch.cuda.device(self.device):
            self._check(self.lib.ncsb_net_infer_stack(
                _ptr(self.params), _ptr(images), T, H, W, _ptr(gamma), per_frame, _ptr(out), sp),
                "ncsb_net_infer_stack")
        return out

    def propose_batch(self, solver, out=None, stream=None):
        """Proposals [solver.batch_tiles, 16, 16] for the batch registered on
        ``solver`` (Solver.batch_set), in the batch's tile order."""
        n = solver.batch_tiles
        if out is None:
            out = torch.empty((n, 16, 16), dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            self._check(self.lib.ncsb_net_infer_batch(
                _ptr(self.params), solver._handle, _ptr(out),
                _stream_ptr(stream, self.device, self.params, out)), "ncsb_net_infer_batch")
        return out

    def propose_stack_tc(self, images, gamma, out=None, stream=None, fp8=False):
        """``propose_stack`` on the tensor cores (BF16 operands, or E4M3 with
        ``fp8``; FP32 accumulation).  Returns (proposals, status) with status
        a one-element int32 device tensor, 1 if a tensor-core wait timed out."""
        T, H, W = images.shape
        per_frame = 1 if gamma.dim() == 3 else 0
        n = _lib.num_tiles(T, H, W)
        if out is None:
            out = torch.empty((n, 16, 16), dtype=torch.float32, device=self.device)
        status = torch.zeros(1, dtype=torch.int32, device=self.device)
        images, gamma = images.contiguous(), gamma.contiguous()
        sp = _stream_ptr(stream, self.device, self.params, images, gamma, out, status)
        name = "ncsb_net_infer_stack_tc_fp8" if fp8 else "ncsb_net_infer_stack_tc"
        with torch.cuda.device(self.device):
            self._check(getattr(self.lib, name)(
                _ptr(self.params), _ptr(images), T, H, W, _ptr(gamma), per_frame, _ptr(out),
                _ptr(status), sp), name)
        return out, status

    def propose_batch_tc(self, solver, out=None, status=None, stream=None, fp8=False):
        """``propose_batch`` on the tensor cores; returns (proposals, status).
        With ``out`` and ``status`` (int32 [1], zeroed by the caller) given,
        one kernel is issued and nothing is allocated, so the call can be
        captured in a CUDA graph; status stays non-zero once a wait times out."""
        n = solver.batch_tiles
        if out is None:
            out = torch.empty((n, 16, 16), dtype=torch.float32, device=self.device)
        if status is None:
            status = torch.zeros(1, dtype=torch.int32, device=self.device)
        name = "ncsb_net_infer_batch_tc_fp8" if fp8 else "ncsb_net_infer_batch_tc"
        with torch.cuda.device(self.device):
            self._check(getattr(self.lib, name)(
                _ptr(self.params), solver._handle, _ptr(out), _ptr(status),
                _stream_ptr(stream, self.device, self.params, out, status)), name)
        return out, status

    def propose_tiles_tc(self, d, gamma, stream=None, fp8=False):
        n = d.shape[0]
        out = torch.empty((n, 16, 16), dtype=torch.float32, device=self.device)
        status = torch.zeros(1, dtype=torch.int32, device=self.device)
        d, gamma = d.contiguous(), gamma.contiguous()
        sp = _stream_ptr(stream, self.device, self.params, d, gamma, out, status)
        name = "ncsb_net_infer_tiles_tc_fp8" if fp8 else "ncsb_net_infer_tiles_tc"
        with torch.cuda.device(self.device):
            self._check(getattr(self.lib, name)(
                _ptr(self.params), _ptr(d), _ptr(gamma), n, _ptr(out), _ptr(status), sp), name)
        return out, status

    def propose_tiles(self, d, gamma, stream=None):
        n = d.shape[0]
        out = torch.empty((n, 16, 16), dtype=torch.float32, device=self.device)
        d, gamma = d.contiguous(), gamma.contiguous()
        sp = _stream_ptr(stream, self.device, self.params, d, gamma, out)
        with torch.cuda.device(self.device):
            self._check(self.lib.ncsb_net_infer_tiles(
                _ptr(self.params), _ptr(d), _ptr(gamma), n, _ptr(out), sp),
                "ncsb_net_infer_tiles")
        return out

    # ---- training -----------------------------------------------------------
    def _buf(self, name, shape, dtype=torch.float32):
        b = self._bufs.get(name)
        if b is None or tuple(b.shape) != tuple(shape):
            b = torch.empty(shape, dtype=dtype, device=self.device)
            self._bufs[name] = b
        return b

    def features(self, d, gamma):
        """Network input [n, 2, 16, 16] and per-tile (mu, s) [n, 2]."""
        n = d.shape[0]
        x = self._buf("x0", (n, 2, 16, 16))
        sc = self._buf("scale", (n, 2))
        with torch.cuda.device(self.device):
            self._check(self.lib.ncsb_net_features(_ptr(d), _ptr(gamma), _ptr(x), _ptr(sc), n,
                                                   _stream_ptr(None, self.device)),
                        "ncsb_net_features")
        return x, sc

    def forward(self, x):
        """Layer outputs [a1, a2, a3, y] of the network on features x."""
        n = x.shape[0]
        acts, cur = [], x
        sp = _stream_ptr(None, self.device)
        for li, ((w, b), (cin, cout, relu)) in enumerate(zip(self._slices(self.params), LAYERS)):
            y = self._buf("a%d" % li, (n, cout, 16, 16))
            self._check(self.lib.ncsb_net_conv_fwd(_ptr(cur), _ptr(w), _ptr(b), _ptr(y), n, cin,
                                                   cout, int(relu), sp), "ncsb_net_conv_fwd")
            acts.append(y)
            cur = y
        return acts

    def loss_and_grad(self, x, target):
        """MSE loss and its gradient [N_PARAMS] for features x and target y*."""
        n = x.shape[0]
        sp = _stream_ptr(None, self.device)
        with torch.cuda.device(self.device):
            acts = self.forward(x)
            grad = self._buf("grad", (N_PARAMS,))
            grad.zero_()
            loss = self._buf("loss", (1,))
            loss.zero_()
            gy = self._buf("g3", (n, 1, 16, 16))
            self._check(self.lib.ncsb_net_mse_grad(_ptr(acts[3]), _ptr(target), _ptr(gy),
                                                   _ptr(loss), n * 256, sp), "ncsb_net_mse_grad")
            gslices = self._slices(grad)
            wslices = self._slices(self.params)
            g = gy
            for li in range(3, -1, -1):
                cin, cout, _ = LAYERS[li]
                inp = acts[li - 1] if li > 0 else x
                dw, db = gslices[li]
                self._check(self.lib.ncsb_net_conv_wgrad(_ptr(inp), _ptr(g), _ptr(dw), _ptr(db),
                                                         n, cin, cout, sp), "ncsb_net_conv_wgrad")
                if li == 0:
                    break
                wf = self._buf("wf%d" % li, (cin * 9 * cout,))
                self._check(self.lib.ncsb_net_flip(_ptr(wslices[li][0]), _ptr(wf), cin, cout, sp),
                            "ncsb_net_flip")
                gx = self._buf("g%d" % (li - 1), (n, cin, 16, 16))
                self._check(self.lib.ncsb_net_conv_fwd(_ptr(g), _ptr(wf), None, _ptr(gx), n, cout,
                                                       cin, 0, sp), "ncsb_net_conv_fwd")
                self._check(self.lib.ncsb_net_relu_bwd(_ptr(gx), _ptr(inp), gx.numel(), sp),
                            "ncsb_net_relu_bwd")
                g = gx
        return loss, grad

    def adam_step(self, grad, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        if self._adam is None:
            self._adam = [torch.zeros_like(self.params), torch.zeros_like(self.params), 0]
        m, v, k = self._adam
        k += 1
        self._adam[2] = k
        with torch.cuda.device(self.device):
            self._check(self.lib.ncsb_net_adam(_ptr(self.params), _ptr(grad), _ptr(m), _ptr(v),
                                               N_PARAMS, lr, b1, b2, eps, k,
                                               _stream_ptr(None, self.device)), "ncsb_net_adam")

    def train(self, d, gamma, u_star, epochs=8, batch=2048, lr=2e-3, lr_final=2e-4, seed=0,
              log=None):
        """Fit the network to converged solutions.  d, gamma, u_star: [N, 16, 16]
        CUDA tensors.  Returns the mean training loss of each epoch."""
        n = d.shape[0]
        x_all = torch.empty((n, 2, 16, 16), dtype=torch.float32, device=self.device)
        t_all = torch.empty((n, 1, 16, 16), dtype=torch.float32, device=self.device)
        for i0 in range(0, n, 65536):
            i1 = min(n, i0 + 65536)
            x, sc = self.features(d[i0:i1].contiguous(), gamma[i0:i1].contiguous())
            x_all[i0:i1] = x
            t_all[i0:i1, 0] = (u_star[i0:i1] - d[i0:i1]) / sc[:, 1].view(-1, 1, 1)
        self._bufs.pop("x0", None)
        gen = torch.Generator(device="cpu")
        gen.manual_seed(seed)
        steps = epochs * max(1, n // batch)
        k, history = 0, []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=gen).to(self.device)
            tot, cnt = torch.zeros((), device=self.device), 0
            for b0 in range(0, n - batch + 1, batch):
                idx = perm[b0:b0 + batch]
                xb = x_all.index_select(0, idx)
                tb = t_all.index_select(0, idx)
                # cosine decay from lr to lr_final
                lr_k = lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * k / steps))
                loss, grad = self.loss_and_grad(xb, tb)
                self.adam_step(grad, lr=lr_k)
                tot += loss[0]
                cnt += 1
                k += 1
            history.append(float(tot) / max(cnt, 1))
            if log:
                log("epoch %d loss %.5f" % (ep, history[-1]))
        return history


# ---- training data ----------------------------------------------------------

def cut_tiles(images, gamma):
    """Tiles [T * tx * ty, 16, 16] of a [T, H, W] stack with the solvers'
    segmentation (origins min(14 i, n + 2 - 16), 1-px edge-replicated halo);
    gamma [H, W] is cut the same way and repeated per frame."""
    T, H, W = images.shape

    def axis(n):
        last, o, out = n + 2 - 16, 0, []
        while True:
            out.append(min(o, last))
            if o >= last:
                break
            o += 14
        idx = torch.tensor([[min(max(b + k - 1, 0), n - 1) for k in range(16)] for b in out],
                           device=images.device)
        return idx

    ri, ci = axis(H), axis(W)
    tx, ty = ri.shape[0], ci.shape[0]

    def cut(a):  # [T, H, W] -> [T, tx, ty, 16, 16]
        rows = a[:, ri.reshape(-1)]                      # [T, tx*16, W]
        blk = rows[:, :, ci.reshape(-1)]                 # [T, tx*16, ty*16]
        return blk.reshape(a.shape[0], tx, 16, ty, 16).permute(0, 1, 3, 2, 4).reshape(-1, 16, 16)

    d = cut(images).contiguous()
    g = cut(gamma.unsqueeze(0)).contiguous()
    g = g.repeat(T, 1, 1) if gamma.dim() == 2 else cut(gamma).contiguous()
    return d, g


def simulate(seed, device, H=512, W=512, frames=3, chains=None):
    """One seeded stack from the training distribution: the full-sensor
    workload's structure density (60 chains per 2048 x 2048 field, so 4 per
    512 x 512) and camera (0.5 % hot pixels with x50 read variance), with
    per-emitter photons U(50, 400) and background U(2, 30) photons/px."""
    from .sim import make_stack_gpu
    rng = numpy.random.default_rng(seed)
    bg = float(rng.uniform(2.0, 30.0))
    if chains is None:
        chains = max(1, int(round(60.0 * H * W / (2048.0 * 2048.0))))
    return make_stack_gpu("sensor2048", T=frames, device=device, seed=int(seed), H=H, W=W,
                          chains=chains, photons=(50.0, 400.0), bg=bg)


def training_tiles(n_tiles, seed=1000, device="cuda", frames=3, log=None):
    """(d, gamma, u_star) [N, 16, 16] from seeded simulations, u_star the plain
    GPU solution at epsilon 1e-6."""
    solver = Solver(alpha=0.2, max_iters=1000, m=4, epsilon=1e-6, mode="plain", device=device)
    ds, gs, us = [], [], []
    have, k = 0, 0
    while have < n_tiles:
        w = simulate(seed + k, device, frames=frames)
        solver.set_otf_mask(w["mask"])
        d, g = cut_tiles(w["images"], w["gamma"])
        u, it, st, _ = solver.solve_tiles(d, g)
        ds.append(d)
        gs.append(g)
        us.append(u)
        have += d.shape[0]
        k += 1
        if log:
            log("simulation %d: %d tiles, mean iters %.1f" % (k, have, it.float().mean().item()))
    d = torch.cat(ds)[:n_tiles].contiguous()
    g = torch.cat(gs)[:n_tiles].contiguous()
    u = torch.cat(us)[:n_tiles].contiguous()
    solver.close()
    return d, g, u


def main():
    ap = argparse.ArgumentParser(description="train the NCS warm-start network on the GPU")
    ap.add_argument("--tiles", type=int, default=200000)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--batch", type=int, default=2048)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1000)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    args = ap.parse_args()
    torch.cuda.init()
    d, g, u = training_tiles(args.tiles, seed=args.seed, log=print)
    net = WarmStartNet(seed=args.seed)
    net.train(d, g, u, epochs=args.epochs, batch=args.batch, lr=args.lr, log=print)
    net.save(args.out)
    print("saved", args.out)


if __name__ == "__main__":
    main()
