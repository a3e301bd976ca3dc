// ncs_norm.cu -- the normalised single-pixel NCS variant
// ("matlab - single pixel with normalization/" in the reference): every pixel
// is its own 3 x 3 segment (the pixel and its 8 neighbours, replicate-padded,
// segpadimg.m with Rs = 1) minimising
//     f(u) = (2/9) sum_i [u_i - c_i log(u_i + gamma_i)] + alpha P(u) / S(u),
//     P(u) = sum_k (|fftshift(fft2(u))_k| / 3 * M_k)^2 = u' Q u,  S(u) = sum_i u_i
// (calcost.m:38-56), from u = d, keeping the segment centre (stitchpadimg.m)
// and setting negative results to 1e-6 (reducenoise.m, optimf).
//
// One thread per pixel: 9 unknowns, FP64 iterate, gradient and costs (the
// cost is a sum of terms of order 100 whose differences near convergence are
// of order 1e-5), BFGS with a dense 9 x 9 inverse-Hessian approximation kept
// in shared memory (45 packed FP32 entries per thread; the direction and the
// update in FP32 as the main solver's L-BFGS, the update's scalars in FP64),
// backtracking Armijo line search on the FP64 cost change (in difference
// form, see the trial loop) with the fraction-to-barrier rule of the main
// solver.  The
// reference minimises with MATLAB's fminunc quasi-Newton; the stopping rule
// here is fminunc's first-order optimality test, ||g||_inf <= tol *
// max(1, ||g_0||_inf), with its iteration cap.  Q (9 x 9, symmetric) is the
// 3 x 3 circular convolution with the kernel qk = ifft2(M^2) / 9 (block
// circulant with circulant blocks): Q[p][q] = qk[(p1 - q1) mod 3][(p2 - q2)
// mod 3], so the kernel takes 9 values from the host instead of 45.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "../../include/ncs_b200.h"

namespace ncsb {
namespace norm {

// 64 threads a block: the inverse Hessians (45 x 4 B a thread) and segment
// constants take 20 KB of static shared memory
constexpr int kThreads = 64;
constexpr int kPacked = 45;  // upper triangle of a symmetric 9 x 9

struct Args {
    const float* data;
    const float* gamma;
    long long gstride;
    float* out;
    int T, H, W;
    double qk[9];  // Q[p][q] = qk[((p/3 - q/3) mod 3) * 3 + (p%3 - q%3) mod 3]
    double alpha, tol, c1, min_step;
    int max_iters;
    int32_t* iters;
    int32_t* status;
    double* cost;
};

__host__ __device__ constexpr int pk(int i, int j) {  // packed index, i <= j
    return i * 9 - i * (i - 1) / 2 + (j - i);
}


// Per-thread constants of the segment in shared memory (c = d + gamma, gamma),
// column t of each [9][kThreads] array.
struct Seg {
    const double (*c)[kThreads];
    const double (*gm)[kThreads];
    int t;
    __device__ double C(int i) const { return c[i][t]; }
    __device__ double G(int i) const { return gm[i][t]; }
};

// Q u, S = sum u and P = u'Q u at a point (the noise term is alpha P / S).
__device__ void noise_parts(const Args& a, const double (&u)[9], double (&Qu)[9], double& S,
                            double& P) {
    S = 0.0;
    P = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        S += u[i];
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < 9; ++j)
            acc = fma(a.qk[((i / 3 - j / 3 + 3) % 3) * 3 + (i % 3 - j % 3 + 3) % 3], u[j], acc);
        Qu[i] = acc;
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) P = fma(u[i], Qu[i], P);
}

// 1/x for x > 0: the hardware's gross FP64 reciprocal (PTX rcp.approx.ftz.f64,
// from the operand's upper 32 bits) refined by two Newton steps r (2 - x r),
// each of which squares the relative error, to FP64 rounding.  No FP32
// round trip: conversions share the pipe with the reciprocal itself.
__device__ __forceinline__ double recip(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    r = r * fma(-x, r, 2.0);
    return r * fma(-x, r, 2.0);
}

// log1p(x) for |x| <= kSeriesMax: 2 atanh(y), y = x / (2 + x), |y| < 0.18, by
// the odd series 2y (1 + y^2/3 + ... + y^14/15); the first omitted term,
// y^16/17, is below 6e-14 relative, and y carries the reciprocal's 2^-46.
constexpr double kSeriesMax = 0.3;
__device__ __forceinline__ double log1p_series(double x) {
    const double y = x * recip(2.0 + x), y2 = y * y;
    double s = fma(y2, 1.0 / 15.0, 1.0 / 13.0);
    s = fma(y2, s, 1.0 / 11.0);
    s = fma(y2, s, 1.0 / 9.0);
    s = fma(y2, s, 1.0 / 7.0);
    s = fma(y2, s, 1.0 / 5.0);
    s = fma(y2, s, 1.0 / 3.0);
    s = fma(y2, s, 1.0);
    return 2.0 * y * s;
}

// the cost at u (FP64 logs; once per pixel, for the reported cost)
__device__ double full_cost(const Args& a, const double (&u)[9], const Seg& sg) {
    double Qu[9], S, P, ll = 0.0;
    noise_parts(a, u, Qu, S, P);
#pragma unroll
    for (int i = 0; i < 9; ++i) ll += u[i] - sg.C(i) * log(u[i] + sg.G(i));
    return (2.0 / 9.0) * ll + a.alpha * P / S;
}

// gradient at u from its noise parts and r_i = 1 / (u_i + gamma_i)
__device__ void gradient(const Args& a, const double (&Qu)[9], double S, double P,
                         const double (&r)[9], const Seg& sg, double (&g)[9]) {
    const double is = recip(S), is2 = is * is;
#pragma unroll
    for (int i = 0; i < 9; ++i)
        g[i] = (2.0 / 9.0) * (1.0 - sg.C(i) * r[i]) + a.alpha * (2.0 * Qu[i] * S - P) * is2;
}

__global__ void __launch_bounds__(kThreads) normalized_kernel(const Args a) {
    __shared__ float Hm[kPacked][kThreads];  // inverse-Hessian approximation, per thread
    __shared__ double Cs[9][kThreads], Gs[9][kThreads];
    __shared__ double Rs[9][kThreads];  // 1 / (u + gamma) at the current iterate
    const long long HW = (long long)a.H * a.W;
    const long long idx = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (idx >= (long long)a.T * HW) return;
    const int f = (int)(idx / HW);
    const long long p = idx - (long long)f * HW;
    const int y = (int)(p / a.W), x = (int)(p - (long long)y * a.W);
    const float* img = a.data + (long long)f * HW;
    const float* gmap = a.gamma + (long long)f * a.gstride;
    const int t = threadIdx.x;
    double u[9], g[9];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const int yy = min(max(y + r - 1, 0), a.H - 1);
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            const int xx = min(max(x + s - 1, 0), a.W - 1);
            const double dv = img[(long long)yy * a.W + xx];
            const double gv = gmap[(long long)yy * a.W + xx];
            u[3 * r + s] = dv;
            Gs[3 * r + s][t] = gv;
            Cs[3 * r + s][t] = dv + gv;
        }
    }
    const Seg sg{Cs, Gs, t};
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
        for (int j = i; j < 9; ++j) Hm[pk(i, j)][t] = i == j ? 1.0f : 0.0f;

    double Qu[9], S, P;
    noise_parts(a, u, Qu, S, P);
    bool feasible = S > 0.0;
    {
        double r[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const double A = u[i] + sg.G(i);
            feasible = feasible && A > 0.0;
            r[i] = recip(A > 0.0 ? A : 1.0);
            Rs[i][t] = r[i];
        }
        gradient(a, Qu, S, P, r, sg, g);
    }
    double fq = feasible ? P * recip(S) : 0.0;  // P / S at the current iterate
    // A trial whose cost change is below the cost's FP64 resolution is accepted,
    // as when two full costs compare equal: near the optimum the gradient still
    // steers the steps (its test can need changes far below that resolution),
    // and a step that moves no pixel ends the solve.  The resolution is taken
    // as 2^-52 of a bound on |f|, (2/9) sum (|u| + c |log(u + gamma)|) +
    // alpha |P / S|, from the start (FP32 hardware log2: only its scale matters)
    double res_f = 0.0;
    if (feasible) {
        float bound = 0.0f;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            float l2;
            asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l2) : "f"((float)(u[i] + sg.G(i))));
            bound += fabsf((float)u[i]) + (float)sg.C(i) * fabsf(l2 * 0.69314718f);
        }
        res_f = 0x1p-52 * ((2.0 / 9.0) * (double)bound + a.alpha * fabs(fq));
    }
    double g0 = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) g0 = fmax(g0, fabs(g[i]));
    int status = NCSB_REACHED_MAXITERS, it = 0;
    if (!feasible) status = NCSB_INCREASING_GRADIENT;  // infeasible start
    for (; it < a.max_iters && status == NCSB_REACHED_MAXITERS; ++it) {
        double gmax = 0.0;
#pragma unroll
        for (int i = 0; i < 9; ++i) gmax = fmax(gmax, fabs(g[i]));
        if (gmax <= a.tol * fmax(1.0, g0)) { status = NCSB_SUCCESS; break; }
        // direction p = -H g and its slope g'p = -g'H g, both FP32 (a quadratic
        // form: no cancellation; the Armijo threshold needs it to 1e-4 at most)
        float d[9];
        double gd;
        float gf[9];
        {
            float gdf = 0.0f;
#pragma unroll
            for (int j = 0; j < 9; ++j) gf[j] = (float)g[j];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                float acc = 0.0f;
#pragma unroll
                for (int j = 0; j < 9; ++j)
                    acc = fmaf(Hm[i <= j ? pk(i, j) : pk(j, i)][t], gf[j], acc);
                d[i] = -acc;
                gdf = fmaf(gf[i], d[i], gdf);
            }
            gd = (double)gdf;
        }
        if (!(gd < 0.0)) {  // lost positive definiteness: restart from steepest descent
#pragma unroll
            for (int i = 0; i < 9; ++i)
#pragma unroll
                for (int j = i; j < 9; ++j) Hm[pk(i, j)][t] = i == j ? 1.0f : 0.0f;
            float gdf = 0.0f;
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                d[i] = -gf[i];
                gdf = fmaf(gf[i], d[i], gdf);
            }
            gd = (double)gdf;
        }
        // backtracking Armijo on the cost change in difference form:
        //   f(un) - f(u) = (2/9) sum_i [s_i - c_i log1p(s_i / (u_i + gamma_i))]
        //                  + alpha (P(un) / S(un) - P(u) / S(u)),  s = un - u,
        // whose log terms are of the order of the step rather than of the costs
        // (about 100), so a series log1p at 1e-13 replaces the FP64 logs of two
        // full costs; trials keep u + gamma >= 1% of its value
        double step = 1.0, un[9], gn[9], Qn[9], Sn = 0.0, Pn = 0.0, fqn = 0.0, df = 0.0;
        bool ok = false;
        for (int trial = 0; trial < 64; ++trial) {
            bool feas = true;
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                un[i] = fma(step, (double)d[i], u[i]);
                feas = feas && (un[i] + sg.G(i) >= 0.01 * (u[i] + sg.G(i)));
            }
            if (feas) {
                noise_parts(a, un, Qn, Sn, Pn);
                if (Sn > 0.0) {
                    double dll = 0.0;
                    bool big = false;
#pragma unroll
                    for (int i = 0; i < 9; ++i) {
                        const double si = un[i] - u[i], x = si * Rs[i][t];
                        big = big || !(fabs(x) <= kSeriesMax);
                        dll += fma(-sg.C(i), log1p_series(x), si);
                    }
                    if (big) {  // a relative step beyond the series' range
                        dll = 0.0;
#pragma unroll
                        for (int i = 0; i < 9; ++i) {
                            const double si = un[i] - u[i];
                            dll += fma(-sg.C(i), log1p(si * Rs[i][t]), si);
                        }
                    }
                    fqn = Pn * recip(Sn);  // the same rounding as fq's
                    df = (2.0 / 9.0) * dll + a.alpha * (fqn - fq);
                    if (df <= a.c1 * step * gd || fabs(df) <= res_f) {
                        ok = true;
                        break;
                    }
                }
            }
            step *= 0.5;
            if (!(step >= a.min_step)) break;
        }
        if (!ok) { status = NCSB_MINIMUM_STEP; break; }
        double rn[9];  // un + gamma >= 1% of u + gamma > 0
#pragma unroll
        for (int i = 0; i < 9; ++i) rn[i] = recip(un[i] + sg.G(i));
        gradient(a, Qn, Sn, Pn, rn, sg, gn);
        // BFGS update of the inverse Hessian with s = un - u, y = gn - g:
        // H <- H - rho (v s' + s v') + (rho^2 y'Hy + rho) s s', v = H y.  The
        // differences and the scalars in FP64, the 45 entries in FP32 from
        // pre-scaled vectors (no FP32 product of rho or rho^2 alone).
        float s[9], yv[9];
        double sy = 0.0, yy = 0.0;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const double sd = un[i] - u[i], yd = gn[i] - g[i];
            s[i] = (float)sd;
            yv[i] = (float)yd;
            sy = fma(sd, yd, sy);
            yy = fma(yd, yd, yy);
        }
        if (sy > 1e-30) {  // rho = 1 / sy within FP32 range
            if (it == 0) {  // scale the identity before the first update
                const float sc = (float)(sy / yy);
#pragma unroll
                for (int i = 0; i < 9; ++i) Hm[pk(i, i)][t] = sc;
            }
            float v[9], yHyf = 0.0f;
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                float acc = 0.0f;
#pragma unroll
                for (int j = 0; j < 9; ++j)
                    acc = fmaf(Hm[i <= j ? pk(i, j) : pk(j, i)][t], yv[j], acc);
                v[i] = acc;
                yHyf = fmaf(yv[i], acc, yHyf);
            }
            const double rho = recip(sy), k2 = rho * rho * (double)yHyf + rho;
            const float rhof = (float)rho;
            float rv[9], ks[9];  // rho v and (rho^2 y'Hy + rho) s (k2 may pass FP32's range)
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                rv[i] = rhof * v[i];
                ks[i] = (float)(k2 * (double)s[i]);
            }
#pragma unroll
            for (int i = 0; i < 9; ++i)
#pragma unroll
                for (int j = i; j < 9; ++j) {
                    const float h = Hm[pk(i, j)][t];
                    Hm[pk(i, j)][t] =
                        fmaf(ks[i], s[j], fmaf(-rv[i], s[j], fmaf(-s[i], rv[j], h)));
                }
        }
        bool moved = false;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            moved = moved || (un[i] != u[i]);
            u[i] = un[i];
            g[i] = gn[i];
            Rs[i][t] = rn[i];
        }
        fq = fqn;
        if (!moved) { status = NCSB_REACHED_MAXPRECISION; ++it; break; }
    }
    const float centre = (float)u[4];
    a.out[idx] = centre < 0.0f ? 1.0e-6f : centre;
    if (a.iters) a.iters[idx] = it;
    if (a.status) a.status[idx] = status;
    if (a.cost) a.cost[idx] = feasible ? full_cost(a, u, sg) : CUDART_INF;
}

}  // namespace norm
}  // namespace ncsb

using namespace ncsb::norm;

extern "C" {

int ncsb_reduce_noise_normalized(const float* images, int n_frames, int height, int width,
                                 const float* gamma, int gamma_per_frame,
                                 const float* mask3_centred, double alpha, int max_iters,
                                 double tolerance, float* out, int32_t* px_iters,
                                 int32_t* px_status, double* px_cost, void* stream) {
    if (!mask3_centred) return NCSB_EINVAL;
    if (n_frames < 0 || height <= 0 || width <= 0 || max_iters < 0) return NCSB_EINVAL;
    if (!(alpha >= 0.0) || !(tolerance >= 0.0)) return NCSB_EINVAL;
    if (n_frames == 0) return NCSB_OK;  // nothing read or written: buffers may be null
    if (!images || !gamma || !out) return NCSB_EINVAL;
    // Q[a][b] = (1/9) sum_k Mu_k^2 Re(conj(F_a[k]) F_b[k]), Mu = ifftshift(mask) (the mask
    // multiplies fftshift(fft2(u))), symmetrised over k -> -k; F_a = fft2 of unit vector a
    double mu[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const double m = mask3_centred[((i + 1) % 3) * 3 + (j + 1) % 3];
            if (!(m == m) || m > 1e300 || m < -1e300) return NCSB_EINVAL;
            mu[i][j] = m * m;
        }
    double sym[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) sym[i][j] = 0.5 * (mu[i][j] + mu[(3 - i) % 3][(3 - j) % 3]);
    Args a{};
    const double tw = 2.0 * 3.14159265358979323846 / 3.0;
    // qk[d1][d2] = Q[(d1, d2)][(0, 0)]; Re(e^{+i th_p} e^{-i th_q}) = cos(th_p - th_q)
    for (int d1 = 0; d1 < 3; ++d1)
        for (int d2 = 0; d2 < 3; ++d2) {
            double acc = 0.0;
            for (int k1 = 0; k1 < 3; ++k1)
                for (int k2 = 0; k2 < 3; ++k2) acc += sym[k1][k2] * cos(tw * (k1 * d1 + k2 * d2));
            a.qk[d1 * 3 + d2] = acc / 9.0;
        }
    a.data = images;
    a.gamma = gamma;
    a.gstride = gamma_per_frame ? (long long)height * width : 0;
    a.out = out;
    a.T = n_frames;
    a.H = height;
    a.W = width;
    a.alpha = alpha;
    a.tol = tolerance;
    a.c1 = 1e-4;
    a.min_step = 1e-12;
    a.max_iters = max_iters;
    a.iters = px_iters;
    a.status = px_status;
    a.cost = px_cost;
    const long long n = (long long)n_frames * height * width;
    normalized_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0,
                        (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

}  // extern "C"
