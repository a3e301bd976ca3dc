"""Python entry points of the B200 NCS solver.

Two layers:

* ``Solver`` -- the torch-level API.  Device tensors in, device tensors out,
  on the caller's current CUDA stream; wraps one ``ncsb_handle``.
* Drop-ins for the reference Python entries, same names, argument meaning and
  error behaviour:
    - ``NCSCUDA`` / ``reduceNoise`` / ``checkOTFMask``  <- cuda/pyCUDANCS/ncs.py:23-226
      (a list of frames + one gamma map + a centred mask; returns a list of
      float32 frames; per-tile failures become ``warnings.warn``)
    - ``cReduceNoise``  <- clib/pyCNCS/ncs_c.py:250-276 (one frame, mask
      already fftshifted; returns float64)
  These take host (numpy) arrays, copy them to the GPU, run the same kernel
  and copy the result back.

All compute runs in libncs_b200.so; there is no CPU fallback.
"""
import ctypes
import warnings

import numpy
import torch

from . import _lib


class NCSCUDAException(Exception):
    """Raised for invalid input in strict mode (cuda/pyCUDANCS/ncs.py:23-24)."""


def checkOTFMask(otf_mask):
    """True when the centred mask has the Hermitian symmetry the cost needs
    (cuda/pyCUDANCS/ncs.py:200-208, clib/pyCNCS/ncs_c.py:239-247)."""
    otf_mask_fft = numpy.fft.ifft2(numpy.fft.fftshift(otf_mask))
    return not (numpy.max(numpy.imag(otf_mask_fft)) > 1.0e-12)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def launch_stream(stream, device, *tensors):
    """The stream a call's kernels run on: ``stream``, else the current one.
    On a caller's stream other than the current one, that stream first waits
    for the current stream (where the wrappers make their contiguous copies
    and allocate their outputs), and every device tensor of the launch is
    recorded on it, so that the caching allocator does not hand their memory
    to other work while the launch may still use it."""
    cur = torch.cuda.current_stream(device)
    if stream is None or stream == cur:
        return cur
    stream.wait_stream(cur)
    for t in tensors:
        if isinstance(t, torch.Tensor) and t.is_cuda:
            t.record_stream(stream)
    return stream


_ADU_TYPES = {torch.float32: _lib.ADU_F32, torch.uint16: _lib.ADU_U16, torch.uint8: _lib.ADU_U8}

_MODES = {"plain": _lib.MODE_PLAIN, "plain_wg": _lib.MODE_PLAIN_WG,
          "spectral": _lib.MODE_SPECTRAL, "tc_tf32": _lib.MODE_TC_TF32,
          "tc_bf16x3": _lib.MODE_TC_BF16X3}


class Solver:
    """One NCS solver handle on one CUDA device.

    Parameters mirror the reference constants (cuda/ncs.cu:54-59): ``alpha``,
    ``max_iters`` (MAXITERS), ``m`` (history size M), ``epsilon`` (stopping
    tolerance on ||g|| / max(1, ||u||)), ``c1`` (Armijo), ``min_step``.
    The default ``epsilon`` is libLBFGS's 1e-5 (the pyCNCS path) rather than
    the reference kernel's 1e-4.  ``mode``: "spectral" (default; L-BFGS with
    the spectral initial inverse Hessian), "plain" (the reference's L-BFGS
    with a scalar initial matrix, one warp per tile), "plain_wg" (one warp
    group per tile), or the tensor-core forms "tc_tf32" and "tc_bf16x3" (the
    spectral algorithm with the noise term's transforms as tcgen05 GEMMs,
    TF32 operands or a three-way BF16 split; m = 1).
    """

    def __init__(self, alpha=0.2, max_iters=200, m=1, epsilon=1e-5, c1=1e-4, min_step=1e-6,
                 mode="spectral", ctas_per_sm=0, device=None):
        self.lib = _lib.load()
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None
                                   else torch.device(device).index or 0)
        self.params = _lib.default_params()
        self._handle = ctypes.c_void_p()
        self._set(alpha=alpha, max_iters=max_iters, m=m, epsilon=epsilon, c1=c1,
                  min_step=min_step, mode=mode, ctas_per_sm=ctas_per_sm)
        with torch.cuda.device(self.device):
            rc = self.lib.ncsb_create(ctypes.byref(self._handle), ctypes.byref(self.params))
        if rc != _lib.NCSB_OK:
            raise RuntimeError("ncsb_create failed with code %d" % rc)
        self.mask_shifted = None

    def _set(self, **kw):
        for k, v in kw.items():
            if k == "mode":
                if v not in _MODES:
                    raise ValueError("unknown mode %r" % (v,))
                v = _MODES[v]
            setattr(self.params, k, v)

    def _check(self, rc):
        if rc != _lib.NCSB_OK:
            msg = self.lib.ncsb_last_error(self._handle).decode()
            if rc == _lib.NCSB_ESIZE:
                raise ValueError(msg)
            raise RuntimeError("libncs_b200 error %d: %s" % (rc, msg))

    def set_params(self, **kw):
        self._set(**kw)
        self._check(self.lib.ncsb_set_params(self._handle, ctypes.byref(self.params)))

    def set_otf_mask_shifted(self, mask_shifted):
        """16x16 mask with DC at [0, 0] (ncs.c / ncs.cu convention)."""
        m = numpy.ascontiguousarray(numpy.asarray(mask_shifted, dtype=numpy.float32))
        if m.shape != (16, 16):
            raise ValueError("OTF mask must be 16 x 16")
        self._check(self.lib.ncsb_set_otf_mask(
            self._handle, m.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        self.mask_shifted = m.copy()

    def set_otf_mask(self, otf_mask_centred):
        """Centred mask (DC in the middle), fftshifted here (ncs.py:197)."""
        self.set_otf_mask_shifted(numpy.fft.fftshift(numpy.asarray(otf_mask_centred)))

    def _tensor(self, x, name, shape=None):
        if not isinstance(x, torch.Tensor) or not x.is_cuda:
            raise TypeError("%s must be a CUDA tensor" % name)
        if x.dtype != torch.float32:
            raise TypeError("%s must be float32" % name)
        if x.device != self.device:
            raise ValueError("%s is on %s, solver on %s" % (name, x.device, self.device))
        if shape is not None and tuple(x.shape) != tuple(shape):
            raise ValueError("%s has shape %s, expected %s" % (name, tuple(x.shape), shape))
        return x.contiguous()

    def num_tiles(self, n_frames, height, width):
        return _lib.num_tiles(n_frames, height, width)

    def reduce_noise(self, images, gamma, out=None, tile_stats=False, stream=None):
        """Denoise a [T, H, W] float32 CUDA stack; gamma is [H, W] (shared) or
        [T, H, W].  Returns ``out`` or, with ``tile_stats``, (out, iters,
        status, cost) where the per-tile arrays follow (frame, row, col) order;
        ``tile_stats="all"`` adds the evaluation counts, and
        ``tile_stats="status"`` returns (out, iters, status) only, without the
        per-tile FP64 cost, whose 256 double-precision logs per tile the
        kernel then skips."""
        images = self._tensor(images, "images")
        if images.dim() == 2:
            images = images.unsqueeze(0)
        T, H, W = images.shape
        gamma = self._tensor(gamma, "gamma")
        if gamma.shape == (H, W):
            per_frame = 0
        elif gamma.shape == (T, H, W):
            per_frame = 1
        else:
            raise ValueError("gamma must be [H, W] or [T, H, W]")
        if out is None:
            out = torch.empty_like(images)
        else:
            out = self._tensor(out, "out", (T, H, W))
        iters = status = cost = evals = None
        if tile_stats:
            n = self.num_tiles(T, H, W)
            iters = torch.empty(n, dtype=torch.int32, device=self.device)
            status = torch.empty(n, dtype=torch.int32, device=self.device)
            if tile_stats != "status":
                cost = torch.empty(n, dtype=torch.float64, device=self.device)
                evals = torch.empty(n, dtype=torch.int32, device=self.device)
        s = launch_stream(stream, self.device, images, gamma, out, iters, status, cost, evals)
        with torch.cuda.device(self.device):
            self._check(self.lib.ncsb_reduce_noise(
                self._handle, _ptr(images), T, H, W, _ptr(gamma), per_frame, _ptr(out),
                _ptr(iters), _ptr(status), _ptr(cost), _ptr(evals),
                ctypes.c_void_p(s.cuda_stream)))
        if tile_stats == "all":
            return out, iters, status, cost, evals
        if tile_stats == "status":
            return out, iters, status
        if tile_stats:
            return out, iters, status, cost
        return out

    def reduce_noise_from(self, images, gamma, u0_tiles, out=None, stream=None, stats=True):
        """reduce_noise starting each tile at a proposal (spectral and tensor-core forms).

        ``u0_tiles`` is [n_tiles, 16, 16] in (frame, tile-row, tile-col) order
        (``WarmStartNet.propose_stack``).  A tile whose proposal costs more
        than its photon image starts at the photon image instead.  Returns
        (out, iters, status, cost, evals, fell_back) with the per-tile arrays
        on the device; fell_back is 1 where the photon-image start was used.
        With ``stats=False`` only (out, fell_back): the kernel then skips the
        per-tile statistics, whose FP64 final cost is a measurable part of a
        solve."""
        images = self._tensor(images, "images")
        T, H, W = images.shape
        gamma = self._tensor(gamma, "gamma")
        if gamma.shape == (H, W):
            per_frame = 0
        elif gamma.shape == (T, H, W):
            per_frame = 1
        else:
            raise ValueError("gamma must be [H, W] or [T, H, W]")
        n = self.num_tiles(T, H, W)
        u0_tiles = self._tensor(u0_tiles, "u0_tiles", (n, 16, 16))
        out = torch.empty_like(images) if out is None else self._tensor(out, "out", (T, H, W))
        iters = status = cost = evals = None
        if stats:
            iters = torch.empty(n, dtype=torch.int32, device=self.device)
            status = torch.empty(n, dtype=torch.int32, device=self.device)
            cost = torch.empty(n, dtype=torch.float64, device=self.device)
            evals = torch.empty(n, dtype=torch.int32, device=self.device)
        start = torch.empty(n, dtype=torch.int32, device=self.device)
        s = launch_stream(stream, self.device, images, gamma, u0_tiles, out, iters, status, cost,
                          evals, start)
        with torch.cuda.device(self.device):
            self._check(self.lib.ncsb_reduce_noise_start(
                self._handle, _ptr(images), T, H, W, _ptr(gamma), per_frame, _ptr(u0_tiles),
                _ptr(out), _ptr(iters), _ptr(status), _ptr(cost), _ptr(evals), _ptr(start),
                ctypes.c_void_p(s.cuda_stream)))
        if not stats:
            return out, start
        return out, iters, status, cost, evals, start

    def _calibration(self, offset, gain, variance, levels, H, W):
        """ncsb_calibration of device maps: offset [H, W], gain and variance
        [H, W] or [L, H, W], L - 1 ascending thresholds."""
        offset = self._tensor(offset, "offset", (H, W))
        gain = self._tensor(gain, "gain")
        variance = self._tensor(variance, "variance")
        if gain.dim() == 2:
            gain = gain.unsqueeze(0)
        if variance.dim() == 2:
            variance = variance.unsqueeze(0)
        L = gain.shape[0]
        if tuple(gain.shape) != (L, H, W) or tuple(variance.shape) != (L, H, W):
            raise ValueError("gain and variance must be [H, W] or [L, H, W] alike")
        if not 1 <= L <= 4 or len(levels) != L - 1:
            raise ValueError("need 1..4 map pairs and one threshold between each two")
        cal = _lib.NcsbCalibration()
        cal.offset, cal.gain, cal.variance = offset.data_ptr(), gain.data_ptr(), variance.data_ptr()
        cal.n_levels = L
        for q, v in enumerate(levels):
            cal.levels[q] = float(v)
        return cal, (offset, gain, variance)

    def reduce_noise_adu(self, adu, offset, gain, variance, levels=(), out=None,
                         tile_stats=False, stream=None):
        """Denoise raw camera frames: ``adu`` [T, H, W] counts (a float32,
        uint16 or uint8 CUDA tensor), ``offset`` [H, W], ``gain`` and
        ``variance`` [H, W] or [L, H, W] (L gain amplifiers, chosen per pixel
        by ADU level against the L - 1 ascending ``levels``).  The conversion
        to photo-electrons (d = (ADU - offset) / gain, non-positive d -> 1e-6,
        gamma = variance / gain^2) is one device pass into a handle-owned
        buffer, then the solve; any solver form.  Integer counts give the same
        result as the same counts in float32.  Returns ``out`` in
        photo-electrons, or with ``tile_stats`` (out, iters, status, cost,
        evals)."""
        if not isinstance(adu, torch.Tensor) or not adu.is_cuda:
            raise TypeError("adu must be a CUDA tensor")
        if adu.dtype not in _ADU_TYPES:
            raise TypeError("adu must be float32, uint16 or uint8")
        if adu.device != self.device:
            raise ValueError("adu is on %s, solver on %s" % (adu.device, self.device))
        adu = adu.contiguous()
        if adu.dim() == 2:
            adu = adu.unsqueeze(0)
        T, H, W = adu.shape
        cal, keep = self._calibration(offset, gain, variance, levels, H, W)
        out = (torch.empty((T, H, W), dtype=torch.float32, device=self.device) if out is None
               else self._tensor(out, "out", (T, H, W)))
        st, cost = [None] * 3, None
        if tile_stats:   # the per-tile FP64 cost is computed only when asked for
            n = self.num_tiles(T, H, W)
            st = [torch.empty(n, dtype=torch.int32, device=self.device) for _ in range(3)]
            cost = torch.empty(n, dtype=torch.float64, device=self.device)
        s = launch_stream(stream, self.device, adu, out, cost, *st, *keep)
        with torch.cuda.device(self.device):
            self._check(self.lib.ncsb_reduce_noise_adu_typed(
                self._handle, _ptr(adu), _ADU_TYPES[adu.dtype], T, H, W, ctypes.byref(cal),
                _ptr(out), _ptr(st[0]), _ptr(st[1]), _ptr(cost), _ptr(st[2]),
                ctypes.c_void_p(s.cuda_stream)))
        if tile_stats:
            return out, st[0], st[1], cost, st[2]
        return out

    def reduce_noise_adu_host(self, adu, offset, gain, variance, levels=(), out=None,
                              chunk_frames=None, n_streams=None, stream=None):
        """Raw frames in host memory to photo-electron results in host memory
        (``ncsb_reduce_noise_adu_host``): ``adu`` [T, H, W] float32, uint16 or
        uint8 (a CPU tensor or numpy array), the calibration maps CUDA
        tensors as in ``reduce_noise_adu``.  Chunks of raw counts are copied
        in, converted, solved and copied out on ``n_streams`` streams, so only
        the camera's own bytes cross the host link inwards.  Page-locked
        ``adu`` and ``out`` give the overlap.  Returns ``out`` (by default a
        new float32 CPU tensor), bit-identical to ``reduce_noise_adu``."""
        h_in = adu if isinstance(adu, torch.Tensor) else torch.from_numpy(numpy.asarray(adu))
        if h_in.device.type != "cpu":
            raise TypeError("reduce_noise_adu_host takes host frames")
        if h_in.dtype not in _ADU_TYPES:
            raise TypeError("adu must be float32, uint16 or uint8")
        h_in = h_in.contiguous()
        if h_in.dim() == 2:
            h_in = h_in.unsqueeze(0)
        if h_in.dim() != 3:
            raise ValueError("adu must be [T, H, W] or [H, W]")
        T, H, W = h_in.shape
        cal, keep = self._calibration(offset, gain, variance, levels, H, W)
        if out is None:
            out = torch.empty((T, H, W), dtype=torch.float32)
        elif (out.device.type != "cpu" or out.dtype != torch.float32
              or tuple(out.shape) != (T, H, W) or not out.is_contiguous()):
            raise ValueError("out must be a contiguous float32 host tensor [T, H, W]")
        s = launch_stream(stream, self.device, *keep)
        with torch.cuda.device(self.device):
            self._check(self.lib.ncsb_reduce_noise_adu_host(
                self._handle, _ptr(h_in), _ADU_TYPES[h_in.dtype], T, H, W, ctypes.byref(cal),
                _ptr(out), int(chunk_frames or 0), int(n_streams or 0),
                ctypes.c_void_p(s.cuda_stream)))
        return out

    # ---- batched launch: many stacks, each with its own alpha and mask ------
    def batch_set(self, stacks):
        """Register a batch of stacks for ``batch_reduce_noise``.  ``stacks`` is
        a sequence of dicts with ``images`` [T, H, W] and ``gamma`` ([H, W] or
        [T, H, W]) float32 CUDA tensors, ``alpha``, and ``mask`` (centred
        16 x 16) or ``mask_shifted``; ``out`` (optional) receives the result
        (allocated here otherwise).  Returns the list of output tensors.  The
        tensors must stay alive while the batch is launched."""
        n = len(stacks)
        if not 1 <= n <= _lib.MAX_STACKS:
            raise ValueError("need 1..%d stacks" % _lib.MAX_STACKS)
        arr = (_lib.NcsbStack * n)()
        keep, outs = [], []
        for i, st in enumerate(stacks):
            images = self._tensor(st["images"], "images")
            if images.dim() == 2:
                images = images.unsqueeze(0)
            T, H, W = images.shape
            gamma = self._tensor(st["gamma"], "gamma")
            if gamma.shape == (H, W):
                per_frame = 0
            elif gamma.shape == (T, H, W):
                per_frame = 1
            else:
                raise ValueError("stack %d: gamma must be [H, W] or [T, H, W]" % i)
            out = st.get("out")
            out = torch.empty_like(images) if out is None else self._tensor(out, "out", (T, H, W))
            a = arr[i]
            a.images, a.gamma, a.out = images.data_ptr(), gamma.data_ptr(), out.data_ptr()
            a.n_frames, a.height, a.width, a.gamma_per_frame = T, H, W, per_frame
            a.alpha = float(st["alpha"])
            if "optics" in st:   # mask built on the device from optics parameters
                a.mask_from_optics = 1
                a.optics = _lib.optics(**st["optics"])
            else:
                if "mask_shifted" in st:
                    ms = numpy.asarray(st["mask_shifted"], dtype=numpy.float32)
                else:
                    ms = numpy.fft.fftshift(numpy.asarray(st["mask"])).astype(numpy.float32)
                if ms.shape != (16, 16):
                    raise ValueError("stack %d: OTF mask must be 16 x 16" % i)
                ctypes.memmove(a.mask_shifted, numpy.ascontiguousarray(ms).ctypes.data, 1024)
            keep.append((images, gamma, out))
            outs.append(out)
        with torch.cuda.device(self.device):
            self._check(self.lib.ncsb_batch_set(self._handle, arr, n))
        self._batch = keep
        n_tiles = ctypes.c_int64(0)
        self._check(self.lib.ncsb_batch_num_tiles(self._handle, ctypes.byref(n_tiles)))
        self.batch_tiles = n_tiles.value
        return outs

    def batch_reduce_noise(self, u0_tiles=None, stats=None, stream=None):
        """Solve the registered batch in one launch.  ``u0_tiles`` (optional,
        [batch_tiles, 16, 16]) are proposed starts; ``stats`` (optional) is a
        dict of preallocated per-tile device tensors with keys among iters,
        status, evals, start (int32) and cost (float64).  Only a counter reset
        and one kernel are issued, so the call can be captured in a CUDA
        graph."""
        if getattr(self, "_batch", None) is None:
            raise RuntimeError("call batch_set first")
        if u0_tiles is not None:
            u0_tiles = self._tensor(u0_tiles, "u0_tiles", (self.batch_tiles, 16, 16))
        st = stats or {}
        s = launch_stream(stream, self.device, u0_tiles, *st.values(),
                          *[t for stack in self._batch for t in stack])
        with torch.cuda.device(self.device):
            self._check(self.lib.ncsb_batch_reduce_noise(
                self._handle, _ptr(u0_tiles), _ptr(st.get("iters")), _ptr(st.get("status")),
                _ptr(st.get("cost")), _ptr(st.get("evals")), _ptr(st.get("start")),
                ctypes.c_void_p(s.cuda_stream)))

    def batch_stats(self):
        """Per-tile device tensors sized for the registered batch."""
        n = self.batch_tiles
        i32 = dict(dtype=torch.int32, device=self.device)
        return {"iters": torch.empty(n, **i32), "status": torch.empty(n, **i32),
                "evals": torch.empty(n, **i32), "start": torch.empty(n, **i32),
                "cost": torch.empty(n, dtype=torch.float64, device=self.device)}

    def reduce_noise_host(self, images, gamma, out=None, chunk_frames=None, n_streams=None,
                          stream=None):
        """Host stack in, host stack out, with the copies hidden behind the solve
        (``ncsb_reduce_noise_host``).

        ``images`` [T, H, W] and ``gamma`` [H, W] or [T, H, W] are float32 CPU
        tensors or numpy arrays.  The library cuts the stack into chunks
        (``chunk_frames`` frames, default T / 40, at most 64 MB); chunk i is
        copied in, solved and copied out on stream i % ``n_streams`` (default
        4), so both directions of the host link and the solve run at once.
        Page-locked inputs and ``out`` (``tensor.pin_memory()``, allocated once
        and reused) give that overlap; pageable memory is accepted as it is
        (the driver stages its copies, which is slower but avoids locking a
        copy of the stack on every call).  Returns ``out`` (by default a new
        float32 CPU tensor), bit-identical to ``reduce_noise``."""
        def host(x):
            t = x if isinstance(x, torch.Tensor) else torch.from_numpy(numpy.asarray(x))
            if t.device.type != "cpu":
                raise TypeError("reduce_noise_host takes host arrays")
            if t.dtype != torch.float32:
                t = t.float()
            return t.contiguous()
        h_in = host(images)
        if h_in.dim() == 2:
            h_in = h_in.unsqueeze(0)
        if h_in.dim() != 3:
            raise ValueError("images must be [T, H, W] or [H, W]")
        T, H, W = h_in.shape
        h_g = host(gamma)
        if tuple(h_g.shape) == (H, W):
            per_frame = 0
        elif tuple(h_g.shape) == (T, H, W):
            per_frame = 1
        else:
            raise ValueError("gamma must be [H, W] or [T, H, W]")
        if out is None:
            out = torch.empty((T, H, W), dtype=torch.float32)
        elif (out.device.type != "cpu" or out.dtype != torch.float32
              or tuple(out.shape) != (T, H, W) or not out.is_contiguous()):
            raise ValueError("out must be a contiguous float32 host tensor [T, H, W]")
        s = launch_stream(stream, self.device)
        with torch.cuda.device(self.device):
            self._check(self.lib.ncsb_reduce_noise_host(
                self._handle, _ptr(h_in), T, H, W, _ptr(h_g), per_frame, _ptr(out),
                int(chunk_frames or 0), int(n_streams or 0), ctypes.c_void_p(s.cuda_stream)))
        return out

    def solve_tiles(self, data, gamma, u0=None, stream=None):
        """Solve [N, 16, 16] tiles (gamma per tile, the layout of the reference
        kernel cuda/ncs.cu:873-879).  Returns (u, iters, status, cost)."""
        data = self._tensor(data, "data")
        n = data.shape[0]
        if tuple(data.shape[1:]) != (16, 16):
            raise ValueError("tiles must be [N, 16, 16]")
        gamma = self._tensor(gamma, "gamma", data.shape)
        if u0 is not None:
            u0 = self._tensor(u0, "u0", data.shape)
        u = torch.empty_like(data)
        iters = torch.empty(n, dtype=torch.int32, device=self.device)
        status = torch.empty(n, dtype=torch.int32, device=self.device)
        cost = torch.empty(n, dtype=torch.float64, device=self.device)
        evals = torch.empty(n, dtype=torch.int32, device=self.device)
        s = launch_stream(stream, self.device, data, gamma, u0, u, iters, status, cost, evals)
        with torch.cuda.device(self.device):
            self._check(self.lib.ncsb_solve_tiles(
                self._handle, _ptr(data), _ptr(gamma), _ptr(u0), n, _ptr(u), _ptr(iters),
                _ptr(status), _ptr(cost), _ptr(evals), ctypes.c_void_p(s.cuda_stream)))
        self.last_evals = evals
        return u, iters, status, cost

    def close(self):
        if getattr(self, "_handle", None) and self._handle.value:
            self.lib.ncsb_destroy(self._handle)
            self._handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _status_report(status, iters, verbose):
    """Warning / verbose summary of per-tile outcomes (cuda/pyCUDANCS/ncs.py:131-159)."""
    status = numpy.asarray(status)
    iters = numpy.asarray(iters)
    failures = {}
    n_fails = int(numpy.count_nonzero(status != 0))
    if n_fails > 0:
        n_maxp = int(numpy.count_nonzero(status == _lib.REACHED_MAXPRECISION))
        if n_maxp != n_fails:
            warnings.warn("Noise reduction failed on {0:d} sub-regions.".format(n_fails))
        for i in range(-5, 0):
            nf = int(numpy.count_nonzero(status == i))
            if nf:
                failures[i] = nf
    if verbose:
        print("Minimum iterations: {0:d}".format(int(iters.min())))
        print("Maximum iterations: {0:d}".format(int(iters.max())))
        print("Median iterations: {0:.3f}".format(float(numpy.median(iters))))
        for key, n in failures.items():
            print(n, "failures of type '" + _lib.STATUS_NAMES[key] + "'")
        print()
    return failures


class NCSCUDA:
    """Drop-in for pyCUDANCS.ncs.NCSCUDA (cuda/pyCUDANCS/ncs.py:27-197).

    ``setOTFMask`` takes the centred 16x16 mask, ``setGamma`` one H x W map
    shared by all frames, ``reduceNoise(images, alpha)`` a list of equally
    sized frames in photo-electrons.  Extra keyword arguments go to
    ``Solver`` (e.g. ``max_iters``, ``epsilon``)."""

    def __init__(self, strict=True, **solver_kwargs):
        self.size = 16
        self.strict = strict
        self.gamma = None
        self.otf_mask = None
        self._solver_kwargs = solver_kwargs
        self._solver = None

    def _get_solver(self, alpha):
        if self._solver is None:
            self._solver = Solver(alpha=float(alpha), **self._solver_kwargs)
        else:
            self._solver.set_params(alpha=float(alpha))
        return self._solver

    def setGamma(self, gamma):
        """CMOS variance / gain^2 in e-^2, shared by all frames (ncs.py:175-181)."""
        self.gamma = numpy.asarray(gamma).astype(numpy.float32)

    def setOTFMask(self, otf_mask):
        """Centred OTF mask (ncs.py:183-197)."""
        otf_mask = numpy.asarray(otf_mask)
        if self.strict:
            if otf_mask.shape[0] != otf_mask.shape[1]:
                raise NCSCUDAException("OTF must be square!")
            if otf_mask.size != self.size * self.size:
                raise NCSCUDAException("OTF size must match sub-region size!")
            if not checkOTFMask(otf_mask):
                raise NCSCUDAException("OTF does not have the expected symmetry!")
        self.otf_mask = numpy.fft.fftshift(otf_mask).astype(numpy.float32)

    def reduceNoise(self, images, alpha, verbose=False):
        """Denoise a list of frames (ncs.py:35-173); returns a list of float32 frames."""
        if self.otf_mask is None or self.gamma is None:
            raise NCSCUDAException("setOTFMask() and setGamma() must be called first")
        images = [numpy.asarray(im) for im in images]
        if len(images) == 0:
            return []
        im0_shape = images[0].shape
        for im in images:
            if im.shape != im0_shape:
                raise NCSCUDAException("All images must be the same size!")
        if self.gamma.shape != im0_shape:
            raise NCSCUDAException("gamma must have the same shape as the images!")
        solver = self._get_solver(alpha)
        solver.set_otf_mask_shifted(self.otf_mask)
        host = torch.from_numpy(numpy.stack(images).astype(numpy.float32)).pin_memory()
        ghost = torch.from_numpy(self.gamma).pin_memory()
        dev = solver.device
        x = host.to(dev, non_blocking=True)
        g = ghost.to(dev, non_blocking=True)
        out, iters, status = solver.reduce_noise(x, g, tile_stats="status")
        result = out.cpu().numpy()
        if verbose:
            print("Processed {0:d} sub-regions.".format(iters.numel()))
        _status_report(status.cpu().numpy(), iters.cpu().numpy(), verbose)
        return [result[i] for i in range(result.shape[0])]


def reduceNoise(images, gamma, otf_mask, alpha, strict=True, verbose=False, **solver_kwargs):
    """Drop-in for pyCUDANCS.ncs.reduceNoise (cuda/pyCUDANCS/ncs.py:211-226)."""
    ncs = NCSCUDA(strict=strict, **solver_kwargs)
    ncs.setOTFMask(otf_mask)
    ncs.setGamma(gamma)
    return ncs.reduceNoise(images, alpha, verbose=verbose)


def cReduceNoise(image, gamma, otf_mask, alpha, strict=True, **solver_kwargs):
    """GPU drop-in for pyCNCS.ncs_c.cReduceNoise (clib/pyCNCS/ncs_c.py:250-276).

    ``otf_mask`` is already fftshifted (DC at [0, 0]), as the reference C call
    expects.  Returns a float64 frame like the reference."""
    otf_mask = numpy.asarray(otf_mask)
    if strict:
        if otf_mask.shape[0] != otf_mask.shape[1]:
            raise NCSCUDAException("OTF must be square!")
        if (otf_mask.shape[0] % 2) != 0:
            raise NCSCUDAException("Sub region size must be divisible by 2!")
    if otf_mask.shape != (16, 16):
        raise NCSCUDAException("Only 16 x 16 sub-regions are supported on the GPU.")
    solver = Solver(alpha=float(alpha), **solver_kwargs)
    solver.set_otf_mask_shifted(otf_mask)
    x = torch.from_numpy(numpy.ascontiguousarray(image, dtype=numpy.float32)).to(solver.device)
    g = torch.from_numpy(numpy.ascontiguousarray(gamma, dtype=numpy.float32)).to(solver.device)
    out = solver.reduce_noise(x, g)
    res = out[0].cpu().numpy().astype(numpy.float64)
    solver.close()
    return res


def reduce_noise_normalized(images, gamma, mask3_centred, alpha=1.0, max_iters=15, tol=1e-6,
                            stats=False, stream=None):
    """The normalised single-pixel variant of NCS (the reference's MATLAB
    package "single pixel with normalization"): 3 x 3 segment per pixel, cost
    2 LL / 9 + alpha NC / sum(u), defaults alpha 1 and 15 iterations as its
    demos.  ``images`` [T, H, W] (or [H, W]) and ``gamma`` ([H, W] or
    [T, H, W]) float32 CUDA tensors; ``mask3_centred`` 3 x 3 (e.g.
    ``otf.normalized_mask()``).  Returns the denoised stack, or with
    ``stats`` (out, iters, status, cost) per pixel."""
    lib = _lib.load()
    if not isinstance(images, torch.Tensor) or not images.is_cuda or images.dtype != torch.float32:
        raise TypeError("images must be a float32 CUDA tensor")
    if images.dim() == 2:
        images = images.unsqueeze(0)
    images = images.contiguous()
    T, H, W = images.shape
    gamma = gamma.contiguous()
    if tuple(gamma.shape) == (H, W):
        per_frame = 0
    elif tuple(gamma.shape) == (T, H, W):
        per_frame = 1
    else:
        raise ValueError("gamma must be [H, W] or [T, H, W]")
    m = numpy.ascontiguousarray(numpy.asarray(mask3_centred, dtype=numpy.float32))
    if m.shape != (3, 3):
        raise ValueError("the normalised variant takes a 3 x 3 mask")
    out = torch.empty_like(images)
    n = T * H * W
    it = st = cost = None
    if stats:
        it = torch.empty(n, dtype=torch.int32, device=images.device)
        st = torch.empty(n, dtype=torch.int32, device=images.device)
        cost = torch.empty(n, dtype=torch.float64, device=images.device)
    s = launch_stream(stream, images.device, images, gamma, out, it, st, cost)
    with torch.cuda.device(images.device):
        rc = lib.ncsb_reduce_noise_normalized(
            _ptr(images), T, H, W, _ptr(gamma), per_frame,
            m.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(alpha), int(max_iters),
            float(tol), _ptr(out), _ptr(it), _ptr(st), _ptr(cost), ctypes.c_void_p(s.cuda_stream))
    if rc != _lib.NCSB_OK:
        raise ValueError("ncsb_reduce_noise_normalized failed with code %d" % rc)
    if stats:
        return out, it.view(T, H, W), st.view(T, H, W), cost.view(T, H, W)
    return out
