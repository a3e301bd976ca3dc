// ncs_plain.cu -- the plain (FP32 SIMT) persistent NCS solver for sm_100a.
//
// One warp group (a 128-thread CTA) solves one 16x16 tile at a time and pulls
// the next tile index from a global atomic counter, so CTAs whose tiles
// converge early keep working.  Per tile it minimises the NCS cost
//     f(u) = sum_i [u_i - c_i log(max(u_i + gamma_i, 1e-6))] + alpha u^T Q u,
//     c_i = d_i + gamma_i,  Q = (1/256) F^H diag(M^2) F
// (clib/pyCNCS/ncs.c:185-299, cuda/ncs.cu:635-817) by L-BFGS with the
// two-loop recursion (ncs.cu:1129-1198) and Armijo backtracking
// (ncs.cu:997-1087), with the reference GPU kernel's stopping rules and
// status codes (ncs.cu:824-852, :1097-1127, :61-67).
//
// Redesign relative to the reference kernel (same iterates in exact
// arithmetic, different cost on the machine):
//  * The noise term is quadratic, so along a search line
//        NC(u + t p) = NC(u) + 2 t p^T Qu + t^2 p^T Qp .
//    Each iteration applies Q once (to the direction p, giving w = Qp) and
//    the line search's trial costs need only the likelihood part; the
//    accepted point's noise gradient is 2 alpha (v + t w) with v = Qu carried
//    along.  The reference does one forward FFT per trial plus an inverse FFT
//    per gradient.
//  * The Armijo test compares the cost DIFFERENCE
//        f(u+tp) - f(u) = sum_i [t p_i - c_i log1p(t p_i / (u_i+gamma_i))]
//                         + alpha (2 t p^T v + t^2 p^T w)
//    evaluated without cancellation and accumulated in FP64, instead of two
//    nearly equal FP32 costs; the convergence test's norms are FP64 too.
//  * Q is applied by an in-register/shared-memory 16x16 FFT: 16-point
//    transforms run across half-warps with shuffles, rows packed two at a
//    time as one complex transform, one shared-memory transpose per pass.
//  * Reductions are warp shuffles plus one named barrier of the warp group.
//  * Tiles are cut from the frame (1-px edge-replicated halo) and stitched
//    back by a closed-form owner rule on the device: frame row y belongs to
//    the last tile (in the reference's row-major order, ncs.c:121-130) whose
//    interior covers it, so every output pixel is written exactly once.
#include "ncs_internal.cuh"

namespace ncsb {

namespace {

struct Smem {
    float2 hs[kMaxM][kThreads];  // L-BFGS s history, thread-ordered pixel pairs
    float2 hy[kMaxM][kThreads];  // L-BFGS y history
    float2 ta[kTile][kTile + 1];  // transpose buffer, forward pass
    float2 tb[kTile][kTile + 1];  // transpose buffer, inverse pass
    double redd[2 * 16];
    float redf[2 * 4];
    long long tile;
};

// y = Q x for the two pixels this thread holds.  x0 = pixel (r, c),
// x1 = pixel (r + 8, c).  msq0/msq1 hold M^2/256 for the spectral positions
// (bitrev(l), g) and (bitrev(l), g + 8) that this thread owns in the column
// pass (g = r, l = c).  Contains two barriers.
__device__ __forceinline__ void apply_q(float x0, float x1, float& y0, float& y1, Smem& sm,
                                        const Twiddles& tw, float msq0, float msq1, int r, int c,
                                        float* nc_part) {
    // Row pass: rows r and r + 8 packed as one complex row.
    float2 z = fft16_fwd(make_float2(x0, x1), c, tw);
    const int k = bitrev4(c);
    const int src = (threadIdx.x & 16) | bitrev4((16 - k) & 15);
    float2 zm;
    zm.x = __shfl_sync(0xffffffffu, z.x, src);
    zm.y = __shfl_sync(0xffffffffu, z.y, src);
    // Z[k] = A[k] + i B[k] with A, B the spectra of the two real rows.
    const float2 A = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
    const float2 B = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
    sm.ta[r][k] = A;
    sm.ta[r + 8][k] = B;
    __syncthreads();
    // Column pass: this thread takes column frequencies g = r and g + 8, row l = c.
    float2 a = sm.ta[c][r];
    float2 b = sm.ta[c][r + 8];
    a = fft16_fwd(a, c, tw);  // now the spectrum at (bitrev(c), r)
    b = fft16_fwd(b, c, tw);  // and at (bitrev(c), r + 8)
    if (nc_part) *nc_part = (a.x * a.x + a.y * a.y) * msq0 + (b.x * b.x + b.y * b.y) * msq1;
    a.x *= msq0; a.y *= msq0;
    b.x *= msq1; b.y *= msq1;
    a = fft16_inv(a, c, tw);  // spatial row c, column frequency r
    b = fft16_inv(b, c, tw);  // spatial row c, column frequency r + 8
    sm.tb[c][r] = a;
    sm.tb[c][r + 8] = b;
    __syncthreads();
    // Row inverse: both output rows are real, so pack them as one transform.
    const float2 e = sm.tb[r][k];
    const float2 f = sm.tb[r + 8][k];
    z = fft16_inv(make_float2(e.x - f.y, e.y + f.x), c, tw);
    y0 = z.x;
    y1 = z.y;
}

}  // namespace

__global__ void __launch_bounds__(kThreads, 8) ncs_plain_kernel(const SolveArgs a) {
    __shared__ Smem sm;
    const int tid = threadIdx.x;
    const int r = tid >> 4, c = tid & 15;
    const Twiddles tw = make_twiddles(c);
    // M^2/256 at the spectral positions (bitrev(c), r) and (bitrev(c), r + 8)
    // this thread owns in the column pass
    const float msq0 = a.msq[bitrev4(c) * 16 + r], msq1 = a.msq[bitrev4(c) * 16 + r + 8];
    const float alpha = a.alpha;
    const int mcap = a.m < 1 ? 1 : (a.m > kMaxM ? kMaxM : a.m);
    int bufd = 0, buff = 0;

    for (;;) {
        if (tid == 0) sm.tile = (long long)atomicAdd(a.queue, 1ull);
        __syncthreads();
        const long long tile = sm.tile;
        if (tile >= a.n_tiles) break;

        // ---- gather the tile (segmentation, ncs.c:66-113) -------------------
        float d0, d1, gm0, gm1, u0, u1;
        int f = 0, ox = 0, oy = 0, own_r = 0, own_c = 0;
        if (a.tile_mode) {
            const long long base = tile * kPix;
            d0 = a.data[base + r * kTile + c];
            d1 = a.data[base + (r + 8) * kTile + c];
            gm0 = a.gamma[base + r * kTile + c];
            gm1 = a.gamma[base + (r + 8) * kTile + c];
            if (a.u0) {
                u0 = a.u0[base + r * kTile + c];
                u1 = a.u0[base + (r + 8) * kTile + c];
            } else {
                u0 = d0;
                u1 = d1;
            }
        } else {
            const long long per_frame = (long long)a.tiles_x * a.tiles_y;
            f = (int)(tile / per_frame);
            const int rem = (int)(tile - (long long)f * per_frame);
            const int ti = rem / a.tiles_y, tj = rem - (rem / a.tiles_y) * a.tiles_y;
            ox = tile_origin(ti, a.H);
            oy = tile_origin(tj, a.W);
            // owned interior: frame rows [ox, next origin) and columns likewise
            own_r = (ti + 1 < a.tiles_x ? tile_origin(ti + 1, a.H) : ox + 14) - ox;
            own_c = (tj + 1 < a.tiles_y ? tile_origin(tj + 1, a.W) : oy + 14) - oy;
            const float* img = a.data + (long long)f * a.H * a.W;
            const float* gmap = a.gamma + (long long)f * a.gamma_frame_stride;
            const int x = clampi(oy + c - 1, 0, a.W - 1);
            const int y0 = clampi(ox + r - 1, 0, a.H - 1);
            const int y1 = clampi(ox + r + 7, 0, a.H - 1);
            d0 = __ldg(img + (long long)y0 * a.W + x);
            d1 = __ldg(img + (long long)y1 * a.W + x);
            gm0 = __ldg(gmap + (long long)y0 * a.W + x);
            gm1 = __ldg(gmap + (long long)y1 * a.W + x);
            u0 = d0;
            u1 = d1;
        }
        const float c0 = d0 + gm0, c1 = d1 + gm1;

        // ---- initial point: v = Q u, g = grad f(u) ------------------------
        float v0, v1;
        apply_q(u0, u1, v0, v1, sm, tw, msq0, msq1, r, c, nullptr);
        float g0 = 1.0f - c0 / fmaxf(u0 + gm0, kFitMin) + 2.0f * alpha * v0;
        float g1 = 1.0f - c1 / fmaxf(u1 + gm1, kFitMin) + 2.0f * alpha * v1;
        int status = kUnstarted, iters = 0, evals = 1;
        {
            double s[2] = {(double)u0 * u0 + (double)u1 * u1, (double)g0 * g0 + (double)g1 * g1};
            block_sum<2>(s, sm.redd, bufd);
            const double unorm = fmax(sqrt(s[0]), 1.0), gnorm = sqrt(s[1]);
            if (gnorm <= (double)a.eps * unorm) status = kSuccess;
            // first direction -g with step 1/||g|| (ncs.cu:980-984)
            float p0 = -g0, p1 = -g1;
            float step = (float)(1.0 / gnorm);
            float rho[kMaxM], al[kMaxM];
            float hscale = 1.0f;
            int nh = 0, newest = -1;

            while (status == kUnstarted) {
                if (iters >= a.max_iters) { status = kReachedMaxIters; break; }
                float w0, w1;
                apply_q(p0, p1, w0, w1, sm, tw, msq0, msq1, r, c, nullptr);
                double q3[3] = {(double)g0 * p0 + (double)g1 * p1,
                                (double)p0 * v0 + (double)p1 * v1,
                                (double)p0 * w0 + (double)p1 * w1};
                block_sum<3>(q3, sm.redd, bufd);
                const double gd = q3[0], pv = q3[1], pw = q3[2];
                if (gd > 0.0) { status = kIncreasingGradient; break; }

                // Armijo backtracking on the exact cost difference.
                const float a0 = u0 + gm0, a1 = u1 + gm1;
                float t = step;
                bool ok = false;
                for (int trial = 0; trial < 64; ++trial) {
                    const float tp0 = t * p0, tp1 = t * p1;
                    const float n0 = a0 + tp0, n1 = a1 + tp1;
                    float l0, l1;
                    if (a0 >= kFitMin && n0 >= kFitMin) l0 = log1pf(tp0 / a0);
                    else l0 = logf(fmaxf(n0, kFitMin)) - logf(fmaxf(a0, kFitMin));
                    if (a1 >= kFitMin && n1 >= kFitMin) l1 = log1pf(tp1 / a1);
                    else l1 = logf(fmaxf(n1, kFitMin)) - logf(fmaxf(a1, kFitMin));
                    // Fraction to the log barrier: a trial that takes a pixel below 1 % of
                    // its u + gamma is infeasible (cost +inf).  Without it the FITMIN
                    // clamp makes points past the barrier look cheaper and Armijo-only
                    // backtracking accepts them (the reference's Moré–Thuente search
                    // rejects them through its curvature test).
                    const bool cross = (a0 >= kFitMin && n0 < kBarrierFrac * a0) ||
                                       (a1 >= kFitMin && n1 < kBarrierFrac * a1);
                    double dl[1] = {cross ? CUDART_INF
                                          : ((double)tp0 - (double)c0 * l0) +
                                                ((double)tp1 - (double)c1 * l1)};
                    block_sum<1>(dl, sm.redd, bufd);
                    ++evals;
                    const double td = (double)t;
                    const double delta = dl[0] + (double)alpha * (2.0 * td * pv + td * td * pw);
                    if (delta <= (double)a.c1 * td * gd) { ok = true; break; }
                    t *= 0.5f;
                    if (!(t >= a.min_step)) break;  // also stops on NaN
                }
                if (!ok) { status = kMinimumStep; break; }  // keep the last good u

                // Accept: u += t p, v += t w, new gradient.
                const float un0 = fmaf(t, p0, u0), un1 = fmaf(t, p1, u1);
                const float vn0 = fmaf(t, w0, v0), vn1 = fmaf(t, w1, v1);
                const float gn0 = 1.0f - c0 / fmaxf(un0 + gm0, kFitMin) + 2.0f * alpha * vn0;
                const float gn1 = 1.0f - c1 / fmaxf(un1 + gm1, kFitMin) + 2.0f * alpha * vn1;
                const float s0 = un0 - u0, s1 = un1 - u1;
                const float y0 = gn0 - g0, y1 = gn1 - g1;
                const int moved = __syncthreads_or((s0 != 0.0f) || (s1 != 0.0f));
                double n4[4] = {(double)un0 * un0 + (double)un1 * un1,
                                (double)gn0 * gn0 + (double)gn1 * gn1,
                                (double)s0 * y0 + (double)s1 * y1,
                                (double)y0 * y0 + (double)y1 * y1};
                block_sum<4>(n4, sm.redd, bufd);
                u0 = un0; u1 = un1; v0 = vn0; v1 = vn1; g0 = gn0; g1 = gn1;
                ++iters;
                if (sqrt(n4[1]) <= (double)a.eps * fmax(sqrt(n4[0]), 1.0)) { status = kSuccess; break; }
                if (!moved) { status = kReachedMaxPrecision; break; }

                // History update (skipped when the curvature pair is unusable).
                const double sy = n4[2], yy = n4[3];
                if (sy > 0.0 && yy > 0.0) {
                    newest = (newest + 1) % mcap;
                    sm.hs[newest][tid] = make_float2(s0, s1);
                    sm.hy[newest][tid] = make_float2(y0, y1);
#pragma unroll
                    for (int i = kMaxM - 1; i > 0; --i) rho[i] = rho[i - 1];
                    rho[0] = (float)(1.0 / sy);
                    hscale = (float)(sy / yy);
                    if (nh < mcap) ++nh;
                }

                // Two-loop recursion: p = -H g.
                float q0 = -g0, q1 = -g1;
#pragma unroll
                for (int i = 0; i < kMaxM; ++i) {
                    if (i < nh) {
                        const int slot = (newest - i + mcap) % mcap;
                        const float2 sv = sm.hs[slot][tid];
                        const float2 yv = sm.hy[slot][tid];
                        const float ai = rho[i] * block_sum_f(sv.x * q0 + sv.y * q1, sm.redf, buff);
                        al[i] = ai;
                        q0 = fmaf(-ai, yv.x, q0);
                        q1 = fmaf(-ai, yv.y, q1);
                    }
                }
                if (nh > 0) {
                    q0 *= hscale;
                    q1 *= hscale;
                }
#pragma unroll
                for (int i = kMaxM - 1; i >= 0; --i) {
                    if (i < nh) {
                        const int slot = (newest - i + mcap) % mcap;
                        const float2 sv = sm.hs[slot][tid];
                        const float2 yv = sm.hy[slot][tid];
                        const float b = rho[i] * block_sum_f(yv.x * q0 + yv.y * q1, sm.redf, buff);
                        q0 = fmaf(al[i] - b, sv.x, q0);
                        q1 = fmaf(al[i] - b, sv.y, q1);
                    }
                }
                p0 = q0;
                p1 = q1;
                if (nh > 0) {
                    step = 1.0f;
                } else {
                    double gg[1] = {(double)g0 * g0 + (double)g1 * g1};
                    block_sum<1>(gg, sm.redd, bufd);
                    step = (float)(1.0 / sqrt(gg[0]));
                }
            }
        }

        // ---- outputs ---------------------------------------------------------
        if (a.cost) {
            const double e0 = (double)u0 - (double)c0 * log(fmax((double)u0 + gm0, 1.0e-6));
            const double e1 = (double)u1 - (double)c1 * log(fmax((double)u1 + gm1, 1.0e-6));
            double fc[2] = {e0 + e1, (double)u0 * v0 + (double)u1 * v1};
            block_sum<2>(fc, sm.redd, bufd);
            if (tid == 0) a.cost[tile] = fc[0] + (double)alpha * fc[1];
        }
        if (tid == 0) {
            if (a.iters) a.iters[tile] = iters;
            if (a.status) a.status[tile] = status;
            if (a.evals) a.evals[tile] = evals;
        }
        if (a.tile_mode) {
            const long long base = tile * kPix;
            a.out[base + r * kTile + c] = u0;
            a.out[base + (r + 8) * kTile + c] = u1;
        } else if (c >= 1 && c <= own_c) {
            float* o = a.out + (long long)f * a.H * a.W;
            const int x = oy + c - 1;
            if (r >= 1 && r <= own_r) o[(long long)(ox + r - 1) * a.W + x] = u0;
            if (r + 8 <= own_r) o[(long long)(ox + r + 7) * a.W + x] = u1;
        }
    }
}

// Host-side launcher.  grid = resident CTAs (persistent).
cudaError_t launch_plain(const SolveArgs& args, int grid, cudaStream_t stream) {
    ncs_plain_kernel<<<grid, kThreads, 0, stream>>>(args);
    return cudaGetLastError();
}

int plain_max_ctas_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ncs_plain_kernel, kThreads, 0) !=
        cudaSuccess)
        return 1;
    return n > 0 ? n : 1;
}

}  // namespace ncsb
