// ncs_warp.cu -- the plain (FP32 SIMT) persistent NCS solver, one warp per
// 16x16 tile.  This is the default form (NCSB_MODE_PLAIN).
//
// It minimises, per tile, the NCS cost
//     f(u) = sum_i [u_i - c_i log(max(u_i + gamma_i, 1e-6))] + alpha u^T Q u,
//     c_i = d_i + gamma_i,  Q = (1/256) F^H diag(M^2) F
// (clib/pyCNCS/ncs.c:185-299, cuda/ncs.cu:635-817) by L-BFGS with up to 8
// correction pairs and Armijo backtracking (ncs.cu:997-1087), with the
// reference GPU kernel's stopping rules and status codes (ncs.cu:824-852,
// :1097-1127, :61-67).  The algorithm is that of ncs_plain.cu (one Q
// application per iteration, FP64 cost-difference Armijo test, fraction-to-
// barrier rule); what changes is the mapping onto the machine:
//
//  * One warp owns a tile and each lane holds 8 pixels, so reductions are
//    warp shuffles only -- no block barrier anywhere in the solve -- and most
//    FFT butterflies are lane-local arithmetic.  A 128-thread CTA holds 4
//    independent warps that pull tiles from the global atomic queue one at a
//    time.  (The warp-group-per-tile kernel of ncs_plain.cu spends ~7,000
//    warp instructions per tile-iteration, mostly in cross-thread traffic;
//    measured and kept for comparison as NCSB_MODE_PLAIN_WG.)
//  * Pixel layout: lane L holds rows P = L >> 2 and P + 8 at columns
//    Qd + 4j (Qd = L & 3, j = 0..3), packed as the complex numbers
//    x[P][c] + i x[P+8][c] -- two real rows per complex transform.
//  * Q x by FFT: 16-point row transforms = lane-local radix-4 step, twiddle,
//    and a 4-point transform across the 4 lanes of a row pair (two shuffle
//    stages with trivial twiddles); one shared-memory transpose; column
//    transforms with 2 lanes per column frequency (the two packed rows are
//    separated lane-locally from X[k] and X[-k], the 16-point column DFT is
//    split into even/odd 8-point DFTs, one per lane); multiply by M^2/256 in
//    that spectral layout; the same steps inverted.
//  * The search direction uses the compact L-BFGS representation (Byrd,
//    Nocedal & Schnabel 1994): all dot products of the new gradient with the
//    stored pairs in one 32-value transposed warp reduction, R and Y'Y from
//    differences of consecutive dot products, the k x k triangular solves on
//    lanes 0..k-1.  Same H g as the two-loop recursion of ncs.cu:1129-1198.
//  * log1p in the line search: 2 atanh(x / (2 + x)) by its odd power series
//    for |x| <= 1/2 (relative error ~1e-7 where the Armijo test needs it),
//    the hardware log2 otherwise.
#include "ncs_warp_common.cuh"

namespace ncsb {

using namespace warp;

// MinBlocks CTAs per SM: the register budget (128 threads each) the
// compiler must meet; the launcher picks the variant shared memory allows.
// MaxM: compiled history capacity (m <= MaxM); a capacity of 4 halves the
// unrolled history loops and the transposed reduction of the default m = 4.
template <int MinBlocks, int MaxM>
__global__ void __launch_bounds__(kWarpCtaThreads, MinBlocks) ncs_warp_kernel(const SolveArgs a) {
    static_assert(MaxM == 4 || MaxM == 8, "history capacity");
    constexpr int NV = (2 * MaxM + 7 <= 16) ? 16 : 32;  // values in the transposed reduction
    constexpr int IA = 0, IB = MaxM, IN = 2 * MaxM;     // slot dots, then the new pair's
    extern __shared__ __align__(16) unsigned char dsm[];
    const int mcap = a.m < 1 ? 1 : (a.m > MaxM ? MaxM : a.m);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float* mtab = reinterpret_cast<float*>(dsm);
    unsigned char* wbase = dsm + kTableBytes + (size_t)wid * warp_bytes(mcap);
    WarpSmem& ws = *reinterpret_cast<WarpSmem*>(wbase);
    float4* hs = reinterpret_cast<float4*>(wbase + ((sizeof(WarpSmem) + 15) / 16) * 16);
    float4* hy = hs + (size_t)mcap * 64;

    // Mask table in the column-pass layout: lane (KC, H), entry i holds
    // M^2/256 at row frequency 2 bitrev3(i) + H, column frequency KC.
    for (int idx = threadIdx.x; idx < 256; idx += blockDim.x) {
        const int L = idx >> 3, i = idx & 7;
        mtab[idx] = a.msq[(2 * bitrev3(i) + (L & 1)) * 16 + (L >> 1)];
    }
    __syncthreads();
    const float* mt = mtab + lane * 8;
    const LaneGeo G = lane_geo(lane);
    const float alpha = a.alpha, two_alpha = 2.0f * a.alpha;

    for (;;) {
        unsigned long long tk = 0;
        if (lane == 0) tk = atomicAdd(a.queue, 1ull);
        const long long tile = (long long)__shfl_sync(kFull, tk, 0);
        if (tile >= a.n_tiles) break;

        // ---- gather the tile (segmentation, ncs.c:66-113) ---------------------
        float d[8], gm[8], u[8];
        int f = 0, ox = 0, oy = 0, own_r = 0, own_c = 0;
        if (a.tile_mode) {
            const long long base = tile * kPix;
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int off = (G.P + 8 * s) * kTile + G.Qd + 4 * j;
                    d[2 * j + s] = __ldg(a.data + base + off);
                    gm[2 * j + s] = __ldg(a.gamma + base + off);
                    u[2 * j + s] = a.u0 ? __ldg(a.u0 + base + off) : d[2 * j + s];
                }
        } else {
            const long long per_frame = (long long)a.tiles_x * a.tiles_y;
            f = (int)(tile / per_frame);
            const int rem = (int)(tile - (long long)f * per_frame);
            const int ti = rem / a.tiles_y, tj = rem - (rem / a.tiles_y) * a.tiles_y;
            ox = tile_origin(ti, a.H);
            oy = tile_origin(tj, a.W);
            own_r = (ti + 1 < a.tiles_x ? tile_origin(ti + 1, a.H) : ox + 14) - ox;
            own_c = (tj + 1 < a.tiles_y ? tile_origin(tj + 1, a.W) : oy + 14) - oy;
            const float* img = a.data + (long long)f * a.H * a.W;
            const float* gmap = a.gamma + (long long)f * a.gamma_frame_stride;
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const long long row = clampi(ox + G.P + 8 * s - 1, 0, a.H - 1);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int col = clampi(oy + G.Qd + 4 * j - 1, 0, a.W - 1);
                    d[2 * j + s] = __ldg(img + row * a.W + col);
                    gm[2 * j + s] = __ldg(gmap + row * a.W + col);
                    u[2 * j + s] = d[2 * j + s];
                }
            }
        }
        float c[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) c[i] = d[i] + gm[i];

        // ---- L-BFGS --------------------------------------------------------------
        // The first pass of the loop applies Q to u (v = Qu, initial gradient);
        // later passes apply it to the direction.  One call site keeps the FFT
        // code once in the instruction stream.
        float v[8], g[8], p[8];
        int status = kUnstarted, iters = 0, evals = 1;
        bool first = true;
        float step = 0.0f;
        int k = 0, head = 0;
        float theta = 1.0f, aold = 0.0f, bold = 0.0f;

        for (;;) {
            if (!first && iters >= a.max_iters) { status = kReachedMaxIters; break; }
            float w[8];
            {
                float xq[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) xq[i] = first ? u[i] : p[i];
                warp_apply_q(xq, w, ws, mt, G, nullptr);
            }
            if (first) {
                first = false;
                float uu = 0.0f, gg = 0.0f;
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    v[i] = w[i];
                    g[i] = 1.0f - __fdividef(c[i], fmaxf(u[i] + gm[i], kFitMin)) + two_alpha * v[i];
                    uu = fmaf(u[i], u[i], uu);
                    gg = fmaf(g[i], g[i], gg);
                    p[i] = -g[i];
                }
                uu = warp_sum_f(uu);
                gg = warp_sum_f(gg);
                if (sqrtf(gg) <= a.eps * fmaxf(sqrtf(uu), 1.0f)) { status = kSuccess; break; }
                step = rsqrtf(gg);  // first step 1/||g|| (ncs.cu:980-984)
                continue;
            }
            float gp = 0.0f, pv = 0.0f, pw = 0.0f;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                gp = fmaf(g[i], p[i], gp);
                pv = fmaf(p[i], v[i], pv);
                pw = fmaf(p[i], w[i], pw);
            }
            const double gd = warp_sum_d((double)gp);
            const double dpv = warp_sum_d((double)pv), dpw = warp_sum_d((double)pw);
            if (gd > 0.0) { status = kIncreasingGradient; break; }

            // Armijo backtracking on the exact cost difference, FP64 across lanes
            float t = step;
            bool ok = false;
            for (int trial = 0; trial < 64; ++trial) {
                float term = 0.0f;
                bool cross = false;
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float ai = u[i] + gm[i];
                    const float tp = t * p[i];
                    const float ni = ai + tp;
                    float l;
                    if (ai >= kFitMin && ni >= kFitMin) l = log1p_ls(__fdividef(tp, ai));
                    else l = __logf(fmaxf(ni, kFitMin)) - __logf(fmaxf(ai, kFitMin));
                    cross |= (ai >= kFitMin) && (ni < kBarrierFrac * ai);
                    term += fmaf(-c[i], l, tp);
                }
                // fraction to the log barrier (see ncs_plain.cu): infeasible trial
                const bool any_cross = __any_sync(kFull, cross);
                const double dl = warp_sum_d((double)term);
                ++evals;
                const double td = (double)t;
                const double delta = any_cross ? CUDART_INF
                                               : dl + (double)alpha * (2.0 * td * dpv + td * td * dpw);
                if (delta <= (double)a.c1 * td * gd) { ok = true; break; }
                t *= 0.5f;
                if (!(t >= a.min_step)) break;  // also stops on NaN
            }
            if (!ok) { status = kMinimumStep; break; }

            // Accept the step; pair s = u_new - u, y = g_new - g.
            float s[8], y[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const float un = fmaf(t, p[i], u[i]);
                v[i] = fmaf(t, w[i], v[i]);
                const float gn = 1.0f - __fdividef(c[i], fmaxf(un + gm[i], kFitMin)) + two_alpha * v[i];
                s[i] = un - u[i];
                y[i] = gn - g[i];
                u[i] = un;
                g[i] = gn;
            }
            // One transposed reduction: s_x'g and y_x'g for the stored slots x, then
            // for the new pair s'g, y'g, s'y, y'y, and ||u||^2, ||g||^2, pixels moved.
            float vals[NV];
#pragma unroll
            for (int i = 0; i < NV; ++i) vals[i] = 0.0f;
#pragma unroll
            for (int x = 0; x < MaxM; ++x) {
                if (x < k) {
                    float hv[8];
                    load8(hs + x * 64 + lane * 2, hv);
                    float acc = 0.0f;
#pragma unroll
                    for (int i = 0; i < 8; ++i) acc = fmaf(hv[i], g[i], acc);
                    vals[IA + x] = acc;
                    load8(hy + x * 64 + lane * 2, hv);
                    acc = 0.0f;
#pragma unroll
                    for (int i = 0; i < 8; ++i) acc = fmaf(hv[i], g[i], acc);
                    vals[IB + x] = acc;
                }
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                vals[IN + 0] = fmaf(s[i], g[i], vals[IN + 0]);
                vals[IN + 1] = fmaf(y[i], g[i], vals[IN + 1]);
                vals[IN + 2] = fmaf(s[i], y[i], vals[IN + 2]);
                vals[IN + 3] = fmaf(y[i], y[i], vals[IN + 3]);
                vals[IN + 4] = fmaf(u[i], u[i], vals[IN + 4]);
                vals[IN + 5] = fmaf(g[i], g[i], vals[IN + 5]);
                vals[IN + 6] += (s[i] != 0.0f) ? 1.0f : 0.0f;
            }
            const float tot = warp_transpose_sum<NV>(vals, lane);  // lane v: total of value v
            const float T16 = __shfl_sync(kFull, tot, IN + 0), T17 = __shfl_sync(kFull, tot, IN + 1);
            const float sy = __shfl_sync(kFull, tot, IN + 2), yy = __shfl_sync(kFull, tot, IN + 3);
            const float un2 = __shfl_sync(kFull, tot, IN + 4), gn2 = __shfl_sync(kFull, tot, IN + 5);
            const float moved = __shfl_sync(kFull, tot, IN + 6);
            const float bnew = __shfl_sync(kFull, tot, IB + (lane & (MaxM - 1)));
            ++iters;
            if (sqrtf(gn2) <= a.eps * fmaxf(sqrtf(un2), 1.0f)) { status = kSuccess; break; }
            if (moved == 0.0f) { status = kReachedMaxPrecision; break; }

            // R_xq = s_x'y_new, (Y'Y)_xq = y_x'y_new from consecutive dot products
            {
                const float rx = tot - aold, tx = bnew - bold;
                aold = tot;  // lanes 0..7: s_x'g of slot x
                bold = bnew;
                if (sy > 0.0f && yy > 0.0f) {
                    const int q = k < mcap ? k : head;  // fresh slot, or evict the oldest
                    store8(hs + q * 64 + lane * 2, s);
                    store8(hy + q * 64 + lane * 2, y);
                    if (lane < k && lane != q) {
                        ws.R[lane][q] = rx;
                        ws.YY[lane][q] = tx;
                        ws.YY[q][lane] = tx;
                    }
                    if (lane == q) {
                        ws.R[q][q] = sy;
                        ws.rinv[q] = 1.0f / sy;
                        ws.YY[q][q] = yy;
                        aold = T16;
                        bold = T17;
                    }
                    if (k < mcap) ++k;
                    else head = head + 1 == mcap ? 0 : head + 1;
                    theta = sy / yy;
                }
            }
            __syncwarp();

            // p = -H g, compact form: H g = theta g + S p1 - theta Y z with
            // z = R^-1 S'g, p1 = R^-T ((D + theta Y'Y) z - theta Y'g); lane j = age j.
            const int j = lane;
            int sj = head + (j & (MaxM - 1));
            if (sj >= mcap) sj -= mcap;
            const float a_slot = __shfl_sync(kFull, aold, sj);
            const float b_slot = __shfl_sync(kFull, bold, sj);
            float zj = 0.0f, p1j = 0.0f, aj = 0.0f, bj = 0.0f;
            if (k > 0) {
                const bool mine = j < k;
                aj = mine ? a_slot : 0.0f;
                bj = mine ? b_slot : 0.0f;
                const float rinv_j = mine ? ws.rinv[sj] : 0.0f;
                float acc = aj;
#pragma unroll
                for (int l = MaxM - 1; l >= 0; --l) {
                    if (l < k) {
                        const float zl = __shfl_sync(kFull, acc * rinv_j, l);
                        int sl = head + l;
                        if (sl >= mcap) sl -= mcap;
                        if (j == l) zj = zl;
                        if (j < l) acc = fmaf(-ws.R[sj][sl], zl, acc);
                    }
                }
                float wsum = 0.0f;
#pragma unroll
                for (int l = 0; l < MaxM; ++l) {
                    if (l < k) {
                        const float zl = __shfl_sync(kFull, zj, l);
                        int sl = head + l;
                        if (sl >= mcap) sl -= mcap;
                        if (mine) wsum = fmaf(ws.YY[sj][sl], zl, wsum);
                    }
                }
                acc = mine ? fmaf(ws.R[sj][sj], zj, theta * (wsum - bj)) : 0.0f;
#pragma unroll
                for (int l = 0; l < MaxM; ++l) {
                    if (l < k) {
                        const float pl = __shfl_sync(kFull, acc * rinv_j, l);
                        int sl = head + l;
                        if (sl >= mcap) sl -= mcap;
                        if (j == l) p1j = pl;
                        if (j > l && mine) acc = fmaf(-ws.R[sl][sj], pl, acc);
                    }
                }
            }
            // g'p from the small quantities; a non-descent direction (rounding)
            // restarts from steepest descent instead of failing
            const float gdl = warp_sum_f(j < k ? fmaf(-p1j, aj, theta * zj * bj) : 0.0f);
            if (k > 0 && !(fmaf(-theta, gn2, gdl) < 0.0f)) {
                k = 0;
                head = 0;
                theta = 1.0f;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) p[i] = -theta * g[i];
#pragma unroll
            for (int l = 0; l < MaxM; ++l) {
                if (l < k) {
                    const float cs = __shfl_sync(kFull, -p1j, l);
                    const float cy = __shfl_sync(kFull, theta * zj, l);
                    int sl = head + l;
                    if (sl >= mcap) sl -= mcap;
                    float hv[8];
                    load8(hs + sl * 64 + lane * 2, hv);
#pragma unroll
                    for (int i = 0; i < 8; ++i) p[i] = fmaf(cs, hv[i], p[i]);
                    load8(hy + sl * 64 + lane * 2, hv);
#pragma unroll
                    for (int i = 0; i < 8; ++i) p[i] = fmaf(cy, hv[i], p[i]);
                }
            }
            step = k > 0 ? 1.0f : rsqrtf(gn2);
        }

        // ---- outputs -----------------------------------------------------------
        if (a.cost) {
            double e0 = 0.0, e1 = 0.0;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                e0 += (double)u[i] - (double)c[i] * log(fmax((double)u[i] + gm[i], 1.0e-6));
                e1 += (double)u[i] * v[i];
            }
            e0 = warp_sum_d(e0);
            e1 = warp_sum_d(e1);
            if (lane == 0) a.cost[tile] = e0 + (double)alpha * e1;
        }
        if (lane == 0) {
            if (a.iters) a.iters[tile] = iters;
            if (a.status) a.status[tile] = status;
            if (a.evals) a.evals[tile] = evals;
        }
        if (a.tile_mode) {
            const long long base = tile * kPix;
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int s = 0; s < 2; ++s)
                    a.out[base + (G.P + 8 * s) * kTile + G.Qd + 4 * j] = u[2 * j + s];
        } else {
            float* o = a.out + (long long)f * a.H * a.W;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int cc = G.Qd + 4 * j;
                if (cc < 1 || cc > own_c) continue;
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int rr = G.P + 8 * s;
                    if (rr >= 1 && rr <= own_r)
                        o[(long long)(ox + rr - 1) * a.W + oy + cc - 1] = u[2 * j + s];
                }
            }
        }
    }
}

size_t warp_smem_bytes(int m) {
    const int mc = m < 1 ? 1 : (m > kMaxM ? kMaxM : m);
    return kTableBytes + (size_t)kWarps * warp_bytes(mc);
}

namespace {

using KernelFn = void (*)(SolveArgs);

template <int MaxM>
KernelFn warp_variant_m(int blocks) {
    switch (blocks <= 3 ? 3 : (blocks >= 6 ? 6 : blocks)) {
        case 3: return ncs_warp_kernel<3, MaxM>;
        case 4: return ncs_warp_kernel<4, MaxM>;
        case 5: return ncs_warp_kernel<5, MaxM>;
        default: return ncs_warp_kernel<6, MaxM>;
    }
}

KernelFn warp_variant(int blocks, int m) {
    return m <= 4 ? warp_variant_m<4>(blocks) : warp_variant_m<8>(blocks);
}

// CTAs per SM that shared memory allows for history size m.
int blocks_by_smem(int m) {
    int dev = 0, per_sm = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) !=
        cudaSuccess)
        per_sm = 228 * 1024;
    const size_t need = warp_smem_bytes(m) + 1024;  // + per-CTA reservation
    return (int)(per_sm / need);
}

}  // namespace

// Default variant: as many CTAs as shared memory allows, at most 4 -- the
// 5- and 6-CTA register budgets (96 / 80) spill and measured slower.
int default_blocks(int m) {
    const int b = blocks_by_smem(m);
    return b < 4 ? b : 4;
}

// Launch with `blocks` CTAs per SM in mind (0 = default_blocks).
cudaError_t launch_warp_blocks(const SolveArgs& args, int grid, int blocks, cudaStream_t stream) {
    const size_t smem = warp_smem_bytes(args.m);
    const KernelFn fn = warp_variant(blocks > 0 ? blocks : default_blocks(args.m), args.m);
    cudaError_t e =
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    fn<<<grid, kWarpCtaThreads, smem, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_warp(const SolveArgs& args, int grid, cudaStream_t stream) {
    return launch_warp_blocks(args, grid, 0, stream);
}

// Resident CTAs per SM of the variant launch_warp_blocks(.., blocks) uses.
int warp_max_ctas_per_sm(int m, int blocks) {
    const size_t smem = warp_smem_bytes(m);
    const KernelFn fn = warp_variant(blocks > 0 ? blocks : default_blocks(m), m);
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return 1;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kWarpCtaThreads, smem) != cudaSuccess)
        return 1;
    return n > 0 ? n : 1;
}

int warp_max_ctas_per_sm(int m) { return warp_max_ctas_per_sm(m, 0); }

}  // namespace ncsb
