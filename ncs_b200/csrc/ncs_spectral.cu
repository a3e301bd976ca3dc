// ncs_spectral.cu -- L-BFGS with a spectral initial inverse Hessian, one warp
// per 16x16 tile (NCSB_MODE_SPECTRAL, the default form).
//
// The per-tile cost (clib/pyCNCS/ncs.c:185-299, cuda/ncs.cu:635-817) has the
// Hessian
//     H = diag(c_i / (u_i + gamma_i)^2) + 2 alpha Q,   Q = (1/256) F^H diag(M^2) F.
// Q is diagonal in Fourier space; only the likelihood part is not.  Replacing
// that diagonal by its tile mean lambda = mean_i c_i / (u_i + gamma_i)^2 gives
//     H0 = (lambda I + 2 alpha Q)^-1 = (1/256) F^H diag(1 / (lambda + 2 alpha M^2)) F,
// which this solver uses as the initial inverse Hessian of the L-BFGS two-loop
// recursion (ncs.cu:1129-1198 uses (s'y / y'y) I), refreshed every iteration.
// On NCS tiles it cuts the iterations to the unchanged stopping rule
// ||g|| <= epsilon max(1, ||u||) about threefold (stack512: 14.6 -> 5.0 mean,
// one line-search trial per iteration), so each solve does less work although
// an iteration now applies two Fourier-diagonal operators:
//   * the first half of the two-loop leaves q; one forward 16x16 FFT of q,
//     the spectral weight 1/(lambda + 2 alpha M^2) and one inverse FFT give
//     H0 q.  Because (lambda + 2 alpha M^2) h = 1 in every bin,
//     2 alpha Q H0 q = q - lambda H0 q needs no transform of its own;
//   * the second half adds coef_i s_i to the direction and coef_i Q s_i to
//     w = 2 alpha Q p, with 2 alpha Q s_i = t_i w_i stored with each pair --
//     so w, which the exact line search needs (ncs_plain.cu), costs no
//     extra transform.  v = 2 alpha Q u is kept the same way.
// Everything else -- FP64 cost-difference Armijo test with the fraction-to-
// barrier rule, stopping rules, status codes, device segmentation and owner-
// rule stitching -- is that of the other solvers.  The first trial step is 1
// (H0 has the right scale); the reference's first step 1/||g||
// (ncs.cu:980-984) compensates for an identity start.
//
// Proposed start (a.u0, tile or stack mode): the first pass transforms the
// proposal u0, which gives an upper bound of f(u0) - f(d) without a transform
// of the photon image d; a proposal the bound accepts starts at once.  Only
// otherwise a second pass transforms d and the solve starts from whichever
// has the lower cost, so a proposal never makes a tile start worse than the
// reference's u = d; the photon-image start is then bit-identical to a solve
// without a proposal.
#include "ncs_warp_common.cuh"

namespace ncsb {

using namespace warp;

namespace {

// Per-warp shared memory: the common block, the s, y and Q s history, then
// the tile's pixel terms c = d + gamma and gamma, then (vg) the vectors v and g.
__host__ __device__ constexpr size_t spec_warp_bytes(int m, bool vg) {
    return ((sizeof(WarpSmem) + 15) / 16) * 16 +
           (3 * (size_t)m + (vg ? 4 : 2)) * 32 * 2 * sizeof(float4);
}

// The 5-CTA launch of the plain single-stack solve keeps v = 2 alpha Q u and
// g in the warp's shared memory instead of registers: at the 96 registers that
// 5 CTAs (20 warps) per SM allow, the solve then runs without spills and
// 0.7 % faster than 4 CTAs with them in registers; at 4 CTAs the extra loads
// measured 0.6 % slower.
template <int MinBlocks, bool Warm, bool Batch>
__host__ __device__ constexpr bool vg_shared() {
    return MinBlocks >= 5 && !Warm && !Batch;
}

// Per-stack pointers and geometry: the kernel parameters of a single-stack
// launch, or the warp's current stack descriptor of a batched one.
struct Geo {
    const float* data;
    const float* gamma;
    float* out;
    long long gstride;
    int H, W, tiles_x, tiles_y;
};

template <bool Batch>
__device__ __forceinline__ Geo geo_of(const SolveArgs& a, const StackDesc& sd) {
    if constexpr (Batch)
        return Geo{sd.data, sd.gamma, sd.out, sd.gamma_frame_stride, sd.H, sd.W, sd.tiles_x,
                   sd.tiles_y};
    else
        return Geo{a.data, a.gamma, a.out, a.gamma_frame_stride, a.H, a.W, a.tiles_x, a.tiles_y};
}

}  // namespace

// Warm: the launch carries proposals (a.u0); the cold variant compiles
// without the start passes.  Batch: tiles of several stacks (own alpha and
// mask each, a.stacks) share one queue; a tile's stack is found by binary
// search over the stacks' first tiles.
template <int MinBlocks, int MaxM, bool Warm, bool Batch>
__global__ void __launch_bounds__(kWarpCtaThreads, MinBlocks) ncs_spectral_kernel(const SolveArgs a) {
    static_assert(MaxM >= 1 && MaxM <= kMaxM, "history capacity");
    extern __shared__ __align__(16) unsigned char dsm[];
    const int mcap = a.m < 1 ? 1 : (a.m > MaxM ? MaxM : a.m);
    // stopping rule ||g|| <= eps max(||u||, 1), compared squared
    const float eps2 = a.eps * a.eps;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    constexpr bool kVg = vg_shared<MinBlocks, Warm, Batch>();
    float* mtab = reinterpret_cast<float*>(dsm);
    unsigned char* wbase = dsm + kTableBytes + (size_t)wid * spec_warp_bytes(mcap, kVg);
    WarpSmem& ws = *reinterpret_cast<WarpSmem*>(wbase);
    float4* hs = reinterpret_cast<float4*>(wbase + ((sizeof(WarpSmem) + 15) / 16) * 16);
    float4* hy = hs + (size_t)mcap * 64;
    float4* hq = hy + (size_t)mcap * 64;
    float4* terms = hq + (size_t)mcap * 64;  // c and gamma, see load_terms
    float4* vbuf = terms + 128;  // kVg: v and g as pixel pairs
    float4* gbuf = terms + 192;

    __shared__ StackDesc sdesc[kWarps];  // Batch: each warp's current stack
    __shared__ TwiddleTable s_tw;
    fill_twiddles(s_tw, threadIdx.x);  // visible after the __syncthreads below
    const LaneGeo G = lane_geo(lane);  // its twiddles are re-read from s_tw
    // M^2/256 at this lane's 8 spectral positions, read once per pass: the
    // CTA's shared table as [half][lane] float4s (conflict-free), or the
    // current stack's table in global memory, lane-major (Batch)
    const float4* mkp = Batch ? nullptr : reinterpret_cast<const float4*>(mtab) + lane;
    float alpha = a.alpha, two_alpha = 2.0f * a.alpha, two_alpha_256 = 512.0f * a.alpha;
    if constexpr (!Batch) {
        for (int idx = threadIdx.x; idx < 256; idx += blockDim.x) {
            const int L = idx >> 3, i = idx & 7;
            mtab[(i >> 2) * 128 + L * 4 + (i & 3)] =
                a.msq[(2 * bitrev3(i) + (L & 1)) * 16 + (L >> 1)];
        }
    }
    __syncthreads();

    for (;;) {
        unsigned long long tk = 0;
        if (lane == 0) tk = atomicAdd(a.queue, 1ull);
        const long long tile = (long long)__shfl_sync(kFull, tk, 0);
        if (tile >= a.n_tiles) break;
        long long lt = tile;  // index of the tile within its stack
        if constexpr (Batch) {
            int lo = 0, hi = a.n_stacks - 1;
            while (lo < hi) {  // last stack whose first tile is <= tile
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(&a.stacks[mid].tile_begin) <= tile) lo = mid;
                else hi = mid - 1;
            }
            __syncwarp();  // every lane is done with the previous tile's descriptor
            if (lane == 0) sdesc[wid] = a.stacks[lo];
            __syncwarp();
            lt = tile - sdesc[wid].tile_begin;
            alpha = sdesc[wid].alpha;
            two_alpha = 2.0f * alpha;
            two_alpha_256 = 512.0f * alpha;
            mkp = reinterpret_cast<const float4*>(a.mk_lane + (size_t)lo * 256) + lane * 2;
        }

        // ---- gather the tile (segmentation, ncs.c:66-113) ---------------------
        // Pixel pairs: element j of a float2[4] holds rows P and P + 8 at column
        // Qd + 4j, the packing of the transforms' complex rows, so that the
        // per-pixel updates run as packed FP32 pairs.
        float d[8], gam[8], u0[8];
        int f = 0, ox = 0, oy = 0, own_r = 0, own_c = 0;
        if (a.tile_mode) {
            const long long base = tile * kPix;
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int off = (G.P + 8 * s) * kTile + G.Qd + 4 * j;
                    d[2 * j + s] = __ldg(a.data + base + off);
                    gam[2 * j + s] = __ldg(a.gamma + base + off);
                    u0[2 * j + s] = Warm ? __ldg(a.u0 + base + off) : d[2 * j + s];
                }
        } else {
            const Geo sg = geo_of<Batch>(a, sdesc[wid]);
            const long long per_frame = (long long)sg.tiles_x * sg.tiles_y;
            f = (int)(lt / per_frame);
            const int rem = (int)(lt - (long long)f * per_frame);
            const int ti = rem / sg.tiles_y, tj = rem - (rem / sg.tiles_y) * sg.tiles_y;
            ox = tile_origin(ti, sg.H);
            oy = tile_origin(tj, sg.W);
            own_r = (ti + 1 < sg.tiles_x ? tile_origin(ti + 1, sg.H) : ox + 14) - ox;
            own_c = (tj + 1 < sg.tiles_y ? tile_origin(tj + 1, sg.W) : oy + 14) - oy;
            const float* img = sg.data + (long long)f * sg.H * sg.W;
            const float* gmap = sg.gamma + (long long)f * sg.gstride;
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const long long row = clampi(ox + G.P + 8 * s - 1, 0, sg.H - 1);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int col = clampi(oy + G.Qd + 4 * j - 1, 0, sg.W - 1);
                    d[2 * j + s] = __ldg(img + row * sg.W + col);
                    gam[2 * j + s] = __ldg(gmap + row * sg.W + col);
                    u0[2 * j + s] = d[2 * j + s];
                }
            }
            if (Warm) {
                const float* ut = a.u0 + tile * kPix;
#pragma unroll
                for (int j = 0; j < 4; ++j)
#pragma unroll
                    for (int s = 0; s < 2; ++s)
                        u0[2 * j + s] = __ldg(ut + (G.P + 8 * s) * kTile + G.Qd + 4 * j);
            }
        }
        float2 u[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) u[j] = make_float2(u0[2 * j], u0[2 * j + 1]);
        // the photon image again, for the start passes of a proposed start
        // (re-read rather than kept in registers through the solve)
        auto load_d = [&](float2 (&dst)[4]) {
            if (a.tile_mode) {
                const float* dt = a.data + tile * kPix;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    dst[j] = make_float2(__ldg(dt + G.P * kTile + G.Qd + 4 * j),
                                         __ldg(dt + (G.P + 8) * kTile + G.Qd + 4 * j));
            } else {
                const Geo sg = geo_of<Batch>(a, sdesc[wid]);
                const float* img = sg.data + (long long)f * sg.H * sg.W;
                const long long r0 = clampi(ox + G.P - 1, 0, sg.H - 1);
                const long long r1 = clampi(ox + G.P + 7, 0, sg.H - 1);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int col = clampi(oy + G.Qd + 4 * j - 1, 0, sg.W - 1);
                    dst[j] = make_float2(__ldg(img + r0 * sg.W + col), __ldg(img + r1 * sg.W + col));
                }
            }
        };
        __syncwarp();  // the previous tile's terms are no longer read
        store_terms_neg(terms, lane, d, gam);
        __syncwarp();

        // ---- preconditioned L-BFGS ---------------------------------------------
        // Pass 0 transforms u (v = 2 alpha Q u, initial gradient); later passes
        // transform the two-loop vector.  One call site for each FFT half.
        // v = 2 alpha Q u carries the factor 2 alpha.  Signs chosen so that the
        // packed updates need no negation: the transformed vector is nq = -q =
        // g + sum a_i y_i (its spectral weights are negated instead), and the
        // solver keeps wn = -w = -2 alpha Q p and the history -Q s; the pixel
        // terms are read as -c (load_terms_neg).
        float2 v[4], g[4], p[4], wn[4];
        // step of each stored pair: its -Q s is kept as t (-Q s) / t = wn, unscaled
        // (t is a power of two, so the scaling is exact either way)
        float rho[MaxM], al[MaxM], tq[MaxM];
        // s'g of the newest pair at the gradient it was stored with: the first
        // two-loop dot of the next iteration, s'(-g), without a reduction
        float sg_newest = 0.0f;
        bool sg_fresh = false;
        int status = kUnstarted, iters = 0, evals = 1, k = 0, newest = -1;
        float lam = 1.0f;
        bool first = true;
        // start passes left: 2 = transform the proposal, then 1 = the photon image
        int start_pass = Warm ? 2 : 0;
        int fell_back = 0;

        for (;;) {
            if (!first && iters >= a.max_iters) { status = kReachedMaxIters; break; }
            float2 nq[4];
            if (first) {
                if (start_pass == 1) {
                    load_d(nq);
                } else {
#pragma unroll
                    for (int j = 0; j < 4; ++j) nq[j] = u[j];
                }
            } else {
                // two-loop, first half (newest pair first), on nq = -q
                if constexpr (kVg) load_hist_volatile(gbuf, lane, g);
#pragma unroll
                for (int j = 0; j < 4; ++j) nq[j] = g[j];
#pragma unroll
                for (int i = 0; i < MaxM; ++i) {
                    if (i < k) {
                        int slot = newest - i;
                        if (slot < 0) slot += mcap;
                        float2 hv[4];
                        float dot;  // s'q
                        if (i == 0 && sg_fresh) {
                            dot = -sg_newest;  // q = -g here
                        } else {
                            load_hist(hs + slot * 64, lane, hv);
                            float2 acc = hv[0] * nq[0];
#pragma unroll
                            for (int e = 1; e < 4; ++e) acc = fma2(hv[e], nq[e], acc);
                            dot = -warp_sum_f(acc.x + acc.y);
                        }
                        const float ai = rho[i] * dot;
                        al[i] = ai;
                        load_hist(hy + slot * 64, lane, hv);
                        const float2 a2 = splat(ai);
#pragma unroll
                        for (int e = 0; e < 4; ++e) nq[e] = fma2(a2, hv[e], nq[e]);
                    }
                }
            }
            // spectral step: p = H0 q (pass 0: 2 alpha Q u) by one forward and
            // one inverse transform; the weights are real and symmetric in k.
            float2 spec[8];
            warp_fft_fwd<false>(nq, spec, ws, with_twiddles(G, s_tw));  // 2 F nq: the weights hold the 1/2
            float mk[8];
            {
                const float4 m0 = Batch ? __ldg(mkp) : mkp[0];
                const float4 m1 = Batch ? __ldg(mkp + 1) : mkp[32];
                mk[0] = m0.x; mk[1] = m0.y; mk[2] = m0.z; mk[3] = m0.w;
                mk[4] = m1.x; mk[5] = m1.y; mk[6] = m1.z; mk[7] = m1.w;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                // -(1/512) / (lam + 512 alpha mk) = 1 / (-512 lam - 512^2 alpha mk): the
                // power-of-two factor moves inside exactly; the sign turns nq into q
                const float wgt = first ? alpha * mk[i]
                                        : rcp_fast(fmaf(-512.0f * two_alpha_256, mk[i], -512.0f * lam));
                spec[i] = make_float2(spec[i].x * wgt, spec[i].y * wgt);
            }
            warp_fft_inv(spec, p, ws, with_twiddles(G, s_tw));
            if (!first) {  // -w = -2 alpha Q H0 q = lambda H0 q - q
                if (two_alpha > 0.0f) {
                    const float2 l2 = splat(lam);
#pragma unroll
                    for (int j = 0; j < 4; ++j) wn[j] = fma2(l2, p[j], nq[j]);
                } else {
#pragma unroll
                    for (int j = 0; j < 4; ++j) wn[j] = make_float2(0.0f, 0.0f);
                }
            }
            if (first) {
                if (start_pass == 2) {
                    // p = v0 = 2 alpha Q u0.  With delta = u0 - d,
                    //   alpha d'Q d = alpha u0'Q u0 - delta'v0 + alpha delta'Q delta
                    //              >= alpha u0'Q u0 - delta'v0,
                    // so f(u0) - f(d) <= LL(u0) - LL(d) + delta'v0: when that
                    // bound is <= 0 the proposal is accepted at once, without
                    // transforming d.  Otherwise keep v0 (in wn) and transform d
                    // next for the exact comparison.
                    float2 dd[4], nc[4], gm[4];
                    load_d(dd);
                    load_terms_neg(terms, lane, nc, gm);
                    float dl = 0.0f, dq = 0.0f;
#pragma unroll
                    for (int j = 0; j < 4; ++j)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const float ui = h ? u[j].y : u[j].x, di = h ? dd[j].y : dd[j].x;
                            const float gi = h ? gm[j].y : gm[j].x, ci = h ? nc[j].y : nc[j].x;
                            const float pi = h ? p[j].y : p[j].x;
                            const float lr = __fsub_rn(__logf(fmaxf(ui + gi, kFitMin)),
                                                       __logf(fmaxf(di + gi, kFitMin)));
                            dl += fmaf(ci, lr, ui - di);
                            dq += __fmul_rn(__fsub_rn(ui, di), pi);
                        }
                    const double bound = warp_sum_d((double)dl + (double)dq);
                    if (bound <= 0.0) {
                        start_pass = 0;  // accepted: v = v0 below
                    } else {
#pragma unroll
                        for (int j = 0; j < 4; ++j) wn[j] = p[j];
                        start_pass = 1;
                        continue;
                    }
                }
                if (start_pass == 1) {
                    // f(u0) - f(d) = sum[(u0 - d) - c (log(u0 + gamma) - log(d + gamma))]
                    //                + alpha (u0'Q u0 - d'Q d);  p = 2 alpha Q d,
                    //                wn = 2 alpha Q u0 here
                    float2 dd[4], nc[4], gm[4];
                    load_d(dd);
                    load_terms_neg(terms, lane, nc, gm);
                    float dl = 0.0f, dq = 0.0f;
#pragma unroll
                    for (int j = 0; j < 4; ++j)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const float ui = h ? u[j].y : u[j].x, di = h ? dd[j].y : dd[j].x;
                            const float gi = h ? gm[j].y : gm[j].x, ci = h ? nc[j].y : nc[j].x;
                            const float pi = h ? p[j].y : p[j].x, wi = h ? wn[j].y : wn[j].x;
                            // explicitly rounded operations: an FMA contraction of
                            // the two logs' scalings, or of the two products, would
                            // leave a rounding residue instead of 0 when u0 = d
                            const float lr = __fsub_rn(__logf(fmaxf(ui + gi, kFitMin)),
                                                       __logf(fmaxf(di + gi, kFitMin)));
                            dl += fmaf(ci, lr, ui - di);
                            dq += __fsub_rn(__fmul_rn(ui, wi), __fmul_rn(di, pi));
                        }
                    const double delta = warp_sum_d((double)dl + 0.5 * (double)dq);
                    if (delta <= 0.0) {
#pragma unroll
                        for (int j = 0; j < 4; ++j) p[j] = wn[j];
                    } else {
                        fell_back = 1;
#pragma unroll
                        for (int j = 0; j < 4; ++j) u[j] = dd[j];
                    }
                    start_pass = 0;
                }
                first = false;
                float2 nc[4], gm[4];
                load_terms_neg(terms, lane, nc, gm);
                float2 uu2 = make_float2(0.0f, 0.0f), gg2 = uu2, ll2 = uu2;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    v[j] = p[j];
                    const float2 A = u[j] + gm[j];
                    const float2 ia = make_float2(rcp_fast(fmaxf(A.x, kFitMin)), rcp_fast(fmaxf(A.y, kFitMin)));
                    const float2 r = nc[j] * ia;  // -c / (u + gamma)
                    g[j] = (r + splat(1.0f)) + v[j];
                    uu2 = fma2(u[j], u[j], uu2);
                    gg2 = fma2(g[j], g[j], gg2);
                    ll2 = fma2(r, ia, ll2);
                }
                if constexpr (kVg) {
                    store_hist(vbuf, lane, v);
                    store_hist(gbuf, lane, g);
                }
                const float uu = warp_sum_f(uu2.x + uu2.y);
                const float gg = warp_sum_f(gg2.x + gg2.y);
                lam = warp_sum_f(ll2.x + ll2.y) * (-1.0f / 256.0f);
                if (gg <= eps2 * fmaxf(uu, 1.0f)) { status = kSuccess; break; }
                continue;
            }
            // two-loop, second half (oldest pair first): p += coef s, wn += coef (-Q s)
#pragma unroll
            for (int i = MaxM - 1; i >= 0; --i) {
                if (i < k) {
                    int slot = newest - i;
                    if (slot < 0) slot += mcap;
                    float2 hv[4];
                    load_hist(hy + slot * 64, lane, hv);
                    float2 acc = hv[0] * p[0];
#pragma unroll
                    for (int e = 1; e < 4; ++e) acc = fma2(hv[e], p[e], acc);
                    const float coef = al[i] - rho[i] * warp_sum_f(acc.x + acc.y);
                    const float2 cf = splat(coef), cq = splat(coef * tq[i]);
                    load_hist(hs + slot * 64, lane, hv);
#pragma unroll
                    for (int e = 0; e < 4; ++e) p[e] = fma2(cf, hv[e], p[e]);
                    load_hist(hq + slot * 64, lane, hv);
#pragma unroll
                    for (int e = 0; e < 4; ++e) wn[e] = fma2(cq, hv[e], wn[e]);
                }
            }

            // this lane's part of the cost change at step t: sum tp - c log1p(tp / A)
            // over its pixels, and whether a pixel crosses the barrier fraction
            auto trial_part = [&](float t, float& part, bool& cross) {
                float2 nc[4], gm[4];
                load_terms_neg(terms, lane, nc, gm);
                const float2 t2 = splat(t);
                float2 term = make_float2(0.0f, 0.0f);
                cross = false;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    // log(max(ni, F)) - log(max(ai, F)) = log1p((max(ni, F) - A) / A),
                    // A = max(ai, F); above the floor the numerator is the exact
                    // step tp (branch free: one select instead of a branch)
                    const float2 ai = u[j] + gm[j];
                    const float2 tp = t2 * p[j];
                    const float2 ni = ai + tp;
                    const float2 bar = splat(kBarrierFrac) * ai;
                    float2 num, rA;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const float a1 = h ? ai.y : ai.x, n1 = h ? ni.y : ni.x;
                        const bool in_dom = a1 >= kFitMin && n1 >= kFitMin;
                        const float A = fmaxf(a1, kFitMin);
                        const float nm = in_dom ? (h ? tp.y : tp.x) : fmaxf(n1, kFitMin) - A;
                        (h ? num.y : num.x) = nm;
                        (h ? rA.y : rA.x) = rcp_fast(A);
                        cross |= (a1 >= kFitMin) && (n1 < (h ? bar.y : bar.x));
                    }
                    term = term + fma2(nc[j], log1p_ls(num * rA), tp);
                }
                part = term.x + term.y;
            };

            // The slopes g'p, p'v, p'w and the first trial's (t = 1) cost change
            // in one FP64 reduction: the trial depends on p alone, and it is
            // accepted in almost every iteration.
            if constexpr (kVg) {
                load_hist_volatile(vbuf, lane, v);
                load_hist_volatile(gbuf, lane, g);
            }
            float2 gp2 = g[0] * p[0], pv2 = p[0] * v[0], pw2 = p[0] * wn[0];
#pragma unroll
            for (int j = 1; j < 4; ++j) {
                gp2 = fma2(g[j], p[j], gp2);
                pv2 = fma2(p[j], v[j], pv2);
                pw2 = fma2(p[j], wn[j], pw2);
            }
            float part0;
            bool cross0;
            trial_part(1.0f, part0, cross0);
            const bool any_cross0 = __any_sync(kFull, cross0);
            double gd = (double)(gp2.x + gp2.y), dpv = (double)(pv2.x + pv2.y),
                   dpw = (double)(pw2.x + pw2.y), dl0 = (double)part0;
            warp_sum4_d(gd, dpv, dpw, dl0, lane);
            dpw = -dpw;  // p'w = -p'wn
            if (!(gd < 0.0)) {
                // not a descent direction: drop the history (H0 alone is positive
                // definite); fail only if even that does not descend
                if (k == 0) { status = kIncreasingGradient; break; }
                k = 0;
                newest = -1;
                sg_fresh = false;
                continue;
            }

            // Armijo backtracking on the exact cost difference, FP64 across lanes
            float t = 1.0f;
            bool ok = false;
            for (int trial = 0; trial < 64; ++trial) {
                double dl = dl0;
                bool any_cross = any_cross0;
                if (trial > 0) {
                    float part;
                    bool cross;
                    trial_part(t, part, cross);
                    any_cross = __any_sync(kFull, cross);
                    dl = warp_sum_d((double)part);
                }
                ++evals;
                const double td = (double)t;
                const double delta = any_cross ? CUDART_INF
                                               : dl + td * dpv + 0.5 * td * td * dpw;
                if (delta <= (double)a.c1 * td * gd) { ok = true; break; }
                t *= 0.5f;
                if (!(t >= a.min_step)) break;  // also stops on NaN
            }
            if (!ok) { status = kMinimumStep; break; }

            // accept; new pair (s, y, -Q s = t wn, stored as wn and t)
            float2 s[4], y[4], nc[4], gm[4];
            load_terms_neg(terms, lane, nc, gm);
            if constexpr (kVg) {
                load_hist_volatile(vbuf, lane, v);
                load_hist_volatile(gbuf, lane, g);
            }
            const float2 t2 = splat(t), z2 = make_float2(0.0f, 0.0f);
            float2 sy2 = z2, uu2 = z2, gg2 = z2, ll2 = z2, mv2 = z2, sg2 = z2;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float2 un = fma2(t2, p[j], u[j]);
                v[j] = fma2(splat(-t), wn[j], v[j]);  // v += t w
                const float2 A = un + gm[j];
                const float2 ia = make_float2(rcp_fast(fmaxf(A.x, kFitMin)), rcp_fast(fmaxf(A.y, kFitMin)));
                const float2 r = nc[j] * ia;  // -c / (u + gamma)
                const float2 gn = (r + splat(1.0f)) + v[j];
                s[j] = un - u[j];
                y[j] = gn - g[j];
                // mv = s's squared norm: zero when no pixel moved (steps below about
                // 1e-22, whose squares underflow, count as none)
                mv2 = fma2(s[j], s[j], mv2);
                u[j] = un;
                g[j] = gn;
                sy2 = fma2(s[j], y[j], sy2);
                sg2 = fma2(s[j], gn, sg2);
                uu2 = fma2(un, un, uu2);
                gg2 = fma2(gn, gn, gg2);
                ll2 = fma2(r, ia, ll2);
            }
            if constexpr (kVg) {
                store_hist(vbuf, lane, v);
                store_hist(gbuf, lane, g);
            }
            float sy, uu, gg, ll, mv, sg;
            {
                float vals[8] = {sy2.x + sy2.y, uu2.x + uu2.y, gg2.x + gg2.y,
                                 ll2.x + ll2.y, mv2.x + mv2.y, sg2.x + sg2.y};
                const float tot = warp_transpose_sum<8>(vals, lane);
                sy = __shfl_sync(kFull, tot, 0);
                uu = __shfl_sync(kFull, tot, 1);
                gg = __shfl_sync(kFull, tot, 2);
                ll = __shfl_sync(kFull, tot, 3);
                mv = __shfl_sync(kFull, tot, 4);
                sg = __shfl_sync(kFull, tot, 5);
            }
            ++iters;
            lam = ll * (-1.0f / 256.0f);
            if (gg <= eps2 * fmaxf(uu, 1.0f)) { status = kSuccess; break; }
            if (mv == 0.0f) { status = kReachedMaxPrecision; break; }
            sg_fresh = sy > 0.0f;
            if (sy > 0.0f) {
                sg_newest = sg;
                newest = newest + 1 == mcap ? 0 : newest + 1;
                store_hist(hs + newest * 64, lane, s);
                store_hist(hy + newest * 64, lane, y);
                store_hist(hq + newest * 64, lane, wn);
#pragma unroll
                for (int i = MaxM - 1; i > 0; --i) {
                    rho[i] = rho[i - 1];
                    tq[i] = tq[i - 1];
                }
                rho[0] = rcp_fast(sy);
                tq[0] = t;
                if (k < mcap) ++k;
            }
        }

        // ---- outputs -----------------------------------------------------------
        if (a.cost) {
            float2 nc[4], gm[4];
            load_terms_neg(terms, lane, nc, gm);
            double e0 = 0.0, e1 = 0.0;
            if constexpr (kVg) load_hist_volatile(vbuf, lane, v);
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const double ui = h ? u[j].y : u[j].x, gi = h ? gm[j].y : gm[j].x;
                    e0 += ui + (double)(h ? nc[j].y : nc[j].x) * log(fmax(ui + gi, 1.0e-6));
                    e1 += ui * (h ? v[j].y : v[j].x);
                }
            e0 = warp_sum_d(e0);
            e1 = warp_sum_d(e1);
            if (lane == 0) a.cost[tile] = e0 + 0.5 * e1;  // v = 2 alpha Q u
        }
        if (lane == 0) {
            if (a.iters) a.iters[tile] = iters;
            if (a.status) a.status[tile] = status;
            if (a.evals) a.evals[tile] = evals;
            if (Warm && a.start) a.start[tile] = fell_back;
        }
        if (a.tile_mode) {
            const long long base = tile * kPix;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                a.out[base + G.P * kTile + G.Qd + 4 * j] = u[j].x;
                a.out[base + (G.P + 8) * kTile + G.Qd + 4 * j] = u[j].y;
            }
        } else {
            const Geo sg = geo_of<Batch>(a, sdesc[wid]);
            float* o = sg.out + (long long)f * sg.H * sg.W;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int cc = G.Qd + 4 * j;
                if (cc < 1 || cc > own_c) continue;
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int rr = G.P + 8 * s;
                    if (rr >= 1 && rr <= own_r)
                        o[(long long)(ox + rr - 1) * sg.W + oy + cc - 1] = s ? u[j].y : u[j].x;
                }
            }
        }
    }
}

namespace {

using KernelFn = void (*)(SolveArgs);

size_t spectral_smem_bytes(int m, bool vg) {
    const int mc = m < 1 ? 1 : (m > 4 ? 4 : m);
    return kTableBytes + (size_t)kWarps * spec_warp_bytes(mc, vg);
}

// whether the instance spectral_variant picks for this launch keeps v and g
// in shared memory (vg_shared above)
bool variant_vg(int blocks, bool warm, bool batch) {
    return blocks >= 5 && !warm && !batch;
}

template <int B, int MaxM>
KernelFn spectral_special(bool warm, bool batch) {
    if (batch) return warm ? ncs_spectral_kernel<B, MaxM, true, true>
                           : ncs_spectral_kernel<B, MaxM, false, true>;
    return ncs_spectral_kernel<B, MaxM, true, false>;
}

template <int MaxM>
KernelFn spectral_variant_m(int blocks, bool warm, bool batch) {
    // proposals and batches: 3 or 4 CTAs per SM
    if (batch || warm)
        return blocks >= 4 ? spectral_special<4, MaxM>(warm, batch)
                           : spectral_special<3, MaxM>(warm, batch);
    switch (blocks <= 3 ? 3 : (blocks >= 5 ? 5 : blocks)) {
        case 3: return ncs_spectral_kernel<3, MaxM, false, false>;
        case 4: return ncs_spectral_kernel<4, MaxM, false, false>;
        default: return ncs_spectral_kernel<5, MaxM, false, false>;
    }
}

KernelFn spectral_variant(int blocks, int m, bool warm, bool batch) {
    return m <= 1 ? spectral_variant_m<1>(blocks, warm, batch)
                  : (m <= 2 ? spectral_variant_m<2>(blocks, warm, batch)
                            : spectral_variant_m<4>(blocks, warm, batch));
}

int spectral_default_blocks(int m, bool warm, bool batch) {
    int dev = 0, per_sm = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) !=
        cudaSuccess)
        per_sm = 228 * 1024;
    // Plain single-stack solves at m = 1: 5 CTAs (20 warps, 96 registers, v and
    // g in shared memory) measured fastest.  Otherwise 4 CTAs (16 warps, 128
    // registers): with more history, proposals or a batch the 5-CTA budget
    // spills.
    if (m <= 1 && !warm && !batch &&
        (int)(per_sm / (spectral_smem_bytes(m, true) + 1024)) >= 5)
        return 5;
    const int b = (int)(per_sm / (spectral_smem_bytes(m, false) + 1024));
    return b < 4 ? b : 4;
}

}  // namespace

cudaError_t launch_spectral(const SolveArgs& args, int grid, int blocks, cudaStream_t stream) {
    const bool warm = args.u0 != nullptr, batch = args.stacks != nullptr;
    const int b = blocks > 0 ? blocks : spectral_default_blocks(args.m, warm, batch);
    const size_t smem = spectral_smem_bytes(args.m, variant_vg(b, warm, batch));
    const KernelFn fn = spectral_variant(b, args.m, warm, batch);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    fn<<<grid, kWarpCtaThreads, smem, stream>>>(args);
    return cudaGetLastError();
}

int spectral_max_ctas_per_sm(int m, int blocks, bool warm, bool batch) {
    const int b = blocks > 0 ? blocks : spectral_default_blocks(m, warm, batch);
    const size_t smem = spectral_smem_bytes(m, variant_vg(b, warm, batch));
    const KernelFn fn = spectral_variant(b, m, warm, batch);
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return 1;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kWarpCtaThreads, smem) != cudaSuccess)
        return 1;
    return n > 0 ? n : 1;
}

}  // namespace ncsb
