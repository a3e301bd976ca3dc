"""Vectorised numpy mirror of the plain GPU solver's algorithm -- TEST
INFRASTRUCTURE ONLY (debugging and iterate-level checks of the CUDA kernel).

It follows ncs_b200/csrc/ncs_plain.cu step by step (one Q-apply per
iteration, FP64 cost-difference Armijo test, two-loop L-BFGS with m pairs,
the reference kernel's stopping rules and status codes of cuda/ncs.cu:61-67),
batched over tiles with per-tile active masks.  Vectors are float32 like the
kernel; Q is applied in FP64 and rounded, so iterates track the kernel
closely but not bit for bit.
"""
import numpy

from .numpy_ref import FITMIN

SUCCESS, MAXITERS, INCREASING, MINSTEP, MAXPREC = 0, -2, -3, -4, -5
BARRIER = 0.01


def apply_q(x, msq):
    """Q x for tiles x [B, 16, 16] (float32 in, float32 out)."""
    y = numpy.real(numpy.fft.ifft2(msq * numpy.fft.fft2(x.astype(numpy.float64))))
    return y.astype(numpy.float32)


def solve(data, gamma, mask_shifted, alpha, max_iters=200, m=8, eps=1e-5, c1=1e-4,
          min_step=1e-6, u0=None, trace=False):
    """Returns (u, iters, status, evals) for tiles [B, 16, 16]."""
    f32 = numpy.float32
    d = numpy.asarray(data, f32)
    gm = numpy.asarray(gamma, f32)
    B = d.shape[0]
    msq = numpy.asarray(mask_shifted, numpy.float64) ** 2
    msq = 0.5 * (msq + numpy.roll(msq[::-1, ::-1], 1, axis=(0, 1)))
    c = (d + gm).astype(f32)
    u = (d if u0 is None else numpy.asarray(u0, f32)).copy()
    al = f32(alpha)
    v = apply_q(u, msq)
    g = (f32(1) - c / numpy.maximum(u + gm, f32(FITMIN)) + f32(2) * al * v).astype(f32)
    status = numpy.full(B, -1, numpy.int32)
    iters = numpy.zeros(B, numpy.int32)
    evals = numpy.ones(B, numpy.int32)
    unorm = numpy.maximum(numpy.sqrt(numpy.sum(u.astype(numpy.float64) ** 2, axis=(1, 2))), 1.0)
    gnorm = numpy.sqrt(numpy.sum(g.astype(numpy.float64) ** 2, axis=(1, 2)))
    status[gnorm <= eps * unorm] = SUCCESS
    p = -g
    step = (1.0 / gnorm).astype(f32)
    S = numpy.zeros((B, m, 16, 16), f32)
    Y = numpy.zeros((B, m, 16, 16), f32)
    rho = numpy.zeros((B, m), f32)
    hscale = numpy.ones(B, f32)
    nh = numpy.zeros(B, numpy.int32)
    newest = numpy.full(B, -1, numpy.int32)
    log = []
    for _ in range(max_iters + 1):
        act = status == -1
        hit = act & (iters >= max_iters)
        status[hit] = MAXITERS
        act = status == -1
        if not act.any():
            break
        w = apply_q(p, msq)
        gd = numpy.sum(g.astype(numpy.float64) * p, axis=(1, 2))
        pv = numpy.sum(p.astype(numpy.float64) * v, axis=(1, 2))
        pw = numpy.sum(p.astype(numpy.float64) * w, axis=(1, 2))
        bad = act & (gd > 0)
        status[bad] = INCREASING
        act &= ~bad
        a = (u + gm).astype(f32)
        t = step.copy()
        ok = numpy.zeros(B, bool)
        searching = act.copy()
        for _trial in range(64):
            if not searching.any():
                break
            tp = (t[:, None, None] * p).astype(f32)
            n = (a + tp).astype(f32)
            regular = (a >= FITMIN) & (n >= FITMIN)
            with numpy.errstate(all="ignore"):
                l_reg = numpy.log1p((tp / a).astype(f32)).astype(f32)
                l_cl = (numpy.log(numpy.maximum(n, f32(FITMIN))).astype(f32)
                        - numpy.log(numpy.maximum(a, f32(FITMIN))).astype(f32))
            lterm = numpy.where(regular, l_reg, l_cl)
            dl = numpy.sum(tp.astype(numpy.float64) - c.astype(numpy.float64) * lterm,
                           axis=(1, 2))
            # fraction to the log barrier: no pixel may lose 99 % of u + gamma
            crossing = numpy.any((a >= FITMIN) & (n < f32(BARRIER) * a), axis=(1, 2))
            dl = numpy.where(crossing, numpy.inf, dl)
            td = t.astype(numpy.float64)
            delta = dl + float(al) * (2.0 * td * pv + td * td * pw)
            evals[searching] += 1
            acc = searching & (delta <= c1 * td * gd)
            ok |= acc
            searching &= ~acc
            t = numpy.where(searching, (t * f32(0.5)).astype(f32), t)
            fail = searching & ~(t >= min_step)
            searching &= ~fail
        fail = act & ~ok
        status[fail] = MINSTEP
        act &= ok
        if trace:
            log.append(dict(t=t.copy(), gd=gd, delta=delta, act=act.copy()))
        T = t[:, None, None]
        un = numpy.where(act[:, None, None], (u + T * p).astype(f32), u)
        vn = numpy.where(act[:, None, None], (v + T * w).astype(f32), v)
        gn = (f32(1) - c / numpy.maximum(un + gm, f32(FITMIN)) + f32(2) * al * vn).astype(f32)
        gn = numpy.where(act[:, None, None], gn, g)
        s = (un - u).astype(f32)
        y = (gn - g).astype(f32)
        moved = numpy.any(s != 0, axis=(1, 2))
        sy = numpy.sum(s.astype(numpy.float64) * y, axis=(1, 2))
        yy = numpy.sum(y.astype(numpy.float64) * y, axis=(1, 2))
        u, v, g = un, vn, gn
        iters[act] += 1
        unorm = numpy.maximum(numpy.sqrt(numpy.sum(u.astype(numpy.float64) ** 2, axis=(1, 2))), 1)
        gnorm = numpy.sqrt(numpy.sum(g.astype(numpy.float64) ** 2, axis=(1, 2)))
        conv = act & (gnorm <= eps * unorm)
        status[conv] = SUCCESS
        act &= ~conv
        prec = act & ~moved
        status[prec] = MAXPREC
        act &= ~prec
        upd = act & (sy > 0) & (yy > 0)
        newest = numpy.where(upd, (newest + 1) % m, newest)
        for b in numpy.nonzero(upd)[0]:
            S[b, newest[b]] = s[b]
            Y[b, newest[b]] = y[b]
            rho[b, 1:] = rho[b, :-1].copy()
            rho[b, 0] = f32(1.0 / sy[b])
            hscale[b] = f32(sy[b] / yy[b])
            nh[b] = min(nh[b] + 1, m)
        q = (-g).astype(f32)
        alph = numpy.zeros((B, m), f32)
        for i in range(m):
            use = act & (i < nh)
            if not use.any():
                continue
            slot = (newest - i) % m
            sv = S[numpy.arange(B), slot]
            yv = Y[numpy.arange(B), slot]
            ai = (rho[:, i] * numpy.sum(sv * q, axis=(1, 2), dtype=numpy.float32)).astype(f32)
            ai = numpy.where(use, ai, f32(0))
            alph[:, i] = ai
            q = (q - ai[:, None, None] * yv).astype(f32)
        q = numpy.where((nh > 0)[:, None, None], (q * hscale[:, None, None]).astype(f32), q)
        for i in range(m - 1, -1, -1):
            use = act & (i < nh)
            if not use.any():
                continue
            slot = (newest - i) % m
            sv = S[numpy.arange(B), slot]
            yv = Y[numpy.arange(B), slot]
            bi = (rho[:, i] * numpy.sum(yv * q, axis=(1, 2), dtype=numpy.float32)).astype(f32)
            coef = numpy.where(use, alph[:, i] - bi, f32(0)).astype(f32)
            q = (q + coef[:, None, None] * sv).astype(f32)
        p = numpy.where(act[:, None, None], q, p)
        gg = numpy.sqrt(numpy.sum(g.astype(numpy.float64) ** 2, axis=(1, 2)))
        step = numpy.where(act, numpy.where(nh > 0, f32(1), (1.0 / gg).astype(f32)), step)
    if trace:
        return u, iters, status, evals, log
    return u, iters, status, evals
