// ncs_net.cu -- kernels of the learned warm start: a 4-layer 3x3 convolutional
// network that maps a tile's photon image and gamma map to a proposed start
// for the L-BFGS solve (include/ncs_b200.h, "learned warm start").  Forward,
// weight gradient, input gradient (forward pass with flipped weights), ReLU
// backward, MSE loss gradient, Adam, and a fused whole-network inference
// kernel that cuts tiles straight from the stack.  FP32 SIMT throughout; one
// 16x16 tile is one image, zero-padded at its border.
//
// Layouts: activations [n][c][16][16] in global memory; in shared memory one
// channel is an 18x18 zero-bordered plane with a channel stride of kCS = 325
// floats (odd, so 32 lanes reading 32 channels at one pixel hit 32 banks);
// weights wt[ci][tap][co], tap = 3 ky + kx, so the outputs of one pixel read
// consecutive weights (float4 broadcasts).
//
// Input features per tile (mu, s = mean and std + 1 of d):
//   x0 = (d - mu) / s,   x1 = sqrt(max(d, 0) + gamma) / s
// and the proposal is u0 = d + s y, clamped to u0 + gamma >= 0.05 max(d + gamma, 1e-3)
// so that the likelihood stays finite at the start.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ncs_b200.h"
#include "ncs_internal.cuh"

namespace ncsb {
namespace net {

constexpr int kPad = 18;  // 16 + 1-px zero border on each side
constexpr int kCS = 325;  // shared-memory channel stride (18 * 18 + 1)
constexpr int kC = 32;    // hidden channels
constexpr int kParams = 2 * 9 * kC + kC + 2 * (kC * 9 * kC + kC) + kC * 9 + 1;
constexpr float kStartFrac = 0.05f;

__host__ __device__ constexpr int round4(int v) { return (v + 3) & ~3; }

// Stage CIN channels of one tile into zero-bordered planes.
template <int CIN>
__device__ __forceinline__ void stage_planes(float* xs, const float* __restrict__ xt) {
    for (int idx = threadIdx.x; idx < CIN * kPad * kPad; idx += blockDim.x) {
        const int ci = idx / (kPad * kPad), rem = idx - ci * (kPad * kPad);
        const int rr = rem / kPad - 1, cc = rem - (rem / kPad) * kPad - 1;
        xs[ci * kCS + rem] =
            (rr >= 0 && rr < 16 && cc >= 0 && cc < 16) ? xt[ci * 256 + rr * 16 + cc] : 0.0f;
    }
}

// acc[co] += sum_ci,tap w[ci][tap][co] x[ci][pixel + tap] for pixel (r, c).
template <int CIN, int COUT>
__device__ __forceinline__ void conv_pixel(const float* xs, const float* ws, int r, int c,
                                           float (&acc)[COUT]) {
    for (int ci = 0; ci < CIN; ++ci) {
        const float* xc = xs + ci * kCS + r * kPad + c;
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) {
            const float xv = xc[(tap / 3) * kPad + tap % 3];
            const float* wr = ws + (ci * 9 + tap) * COUT;
            if constexpr (COUT % 4 == 0) {
#pragma unroll
                for (int q = 0; q < COUT / 4; ++q) {
                    const float4 w4 = reinterpret_cast<const float4*>(wr)[q];
                    acc[4 * q + 0] = fmaf(w4.x, xv, acc[4 * q + 0]);
                    acc[4 * q + 1] = fmaf(w4.y, xv, acc[4 * q + 1]);
                    acc[4 * q + 2] = fmaf(w4.z, xv, acc[4 * q + 2]);
                    acc[4 * q + 3] = fmaf(w4.w, xv, acc[4 * q + 3]);
                }
            } else {
#pragma unroll
                for (int co = 0; co < COUT; ++co) acc[co] = fmaf(wr[co], xv, acc[co]);
            }
        }
    }
}

// y = conv3x3(x) + b (optionally ReLU).  One CTA (256 threads) per tile, one
// thread per pixel.
template <int CIN, int COUT, bool RELU>
__global__ void __launch_bounds__(256) conv3x3_fwd(const float* __restrict__ x,
                                                   const float* __restrict__ wt,
                                                   const float* __restrict__ b,
                                                   float* __restrict__ y, int n) {
    extern __shared__ __align__(16) float sm[];
    float* xs = sm;
    float* ws = sm + round4(CIN * kCS);
    const int tile = blockIdx.x;
    if (tile >= n) return;
    const int p = threadIdx.x, r = p >> 4, c = p & 15;
    stage_planes<CIN>(xs, x + (size_t)tile * CIN * 256);
    for (int idx = threadIdx.x; idx < CIN * 9 * COUT; idx += 256) ws[idx] = wt[idx];
    __syncthreads();
    float acc[COUT];
#pragma unroll
    for (int co = 0; co < COUT; ++co) acc[co] = b ? b[co] : 0.0f;
    conv_pixel<CIN, COUT>(xs, ws, r, c, acc);
    float* yt = y + (size_t)tile * COUT * 256;
#pragma unroll
    for (int co = 0; co < COUT; ++co) yt[co * 256 + p] = RELU ? fmaxf(acc[co], 0.0f) : acc[co];
}

// dwt[ci][tap][co] += sum_tiles,pixels dy[co][p] x[ci][p + tap], db += sum dy.
// Thread (ps, ci, g) owns the 9 x CO_PER weights of input channel ci and
// output channels g*CO_PER.. and walks the rows ps, ps + PS, ... of each tile
// with a sliding 3x3 window: per pixel 3 new x values, CO_PER dy values and
// 9 CO_PER FMAs.  Partial sums go to global memory with one atomicAdd per
// weight per thread at the end.
template <int CIN, int COUT>
__global__ void __launch_bounds__(256) conv3x3_wgrad(const float* __restrict__ x,
                                                     const float* __restrict__ dy,
                                                     float* __restrict__ dwt,
                                                     float* __restrict__ db, int n, int per_cta) {
    constexpr int CO_PER = COUT >= 4 ? 4 : COUT;
    constexpr int NG = COUT / CO_PER;
    constexpr int LANES = CIN * NG;
    constexpr int PS = 256 / LANES;
    static_assert(COUT % CO_PER == 0 && 256 % LANES == 0 && PS >= 1 && PS <= 16, "mapping");
    constexpr int GS = 257;  // dy channel stride in shared memory
    extern __shared__ __align__(16) float sm[];
    float* xs = sm;
    float* gs = sm + round4(CIN * kCS);
    const int t = threadIdx.x;
    const int g = t % NG, ci = (t / NG) % CIN, ps = t / LANES;
    float acc[9][CO_PER], bacc[CO_PER];
#pragma unroll
    for (int k = 0; k < 9; ++k)
#pragma unroll
        for (int j = 0; j < CO_PER; ++j) acc[k][j] = 0.0f;
#pragma unroll
    for (int j = 0; j < CO_PER; ++j) bacc[j] = 0.0f;

    const int t0 = blockIdx.x * per_cta;
    const int t1 = min(t0 + per_cta, n);
    for (int tile = t0; tile < t1; ++tile) {
        __syncthreads();  // the previous tile's planes are no longer read
        stage_planes<CIN>(xs, x + (size_t)tile * CIN * 256);
        const float* gt = dy + (size_t)tile * COUT * 256;
        for (int idx = threadIdx.x; idx < COUT * 256; idx += 256)
            gs[(idx >> 8) * GS + (idx & 255)] = gt[idx];
        __syncthreads();
        const float* xc = xs + ci * kCS;
        for (int r = ps; r < 16; r += PS) {
            float win[3][3];
#pragma unroll
            for (int ky = 0; ky < 3; ++ky) {
                win[ky][0] = xc[(r + ky) * kPad + 0];
                win[ky][1] = xc[(r + ky) * kPad + 1];
            }
#pragma unroll
            for (int c = 0; c < 16; ++c) {
#pragma unroll
                for (int ky = 0; ky < 3; ++ky) win[ky][2] = xc[(r + ky) * kPad + c + 2];
                float dv[CO_PER];
#pragma unroll
                for (int j = 0; j < CO_PER; ++j) dv[j] = gs[(g * CO_PER + j) * GS + r * 16 + c];
#pragma unroll
                for (int ky = 0; ky < 3; ++ky)
#pragma unroll
                    for (int kx = 0; kx < 3; ++kx)
#pragma unroll
                        for (int j = 0; j < CO_PER; ++j)
                            acc[ky * 3 + kx][j] = fmaf(win[ky][kx], dv[j], acc[ky * 3 + kx][j]);
#pragma unroll
                for (int j = 0; j < CO_PER; ++j) bacc[j] += dv[j];
#pragma unroll
                for (int ky = 0; ky < 3; ++ky) {
                    win[ky][0] = win[ky][1];
                    win[ky][1] = win[ky][2];
                }
            }
        }
    }
    if (t1 <= t0) return;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap)
#pragma unroll
        for (int j = 0; j < CO_PER; ++j)
            atomicAdd(dwt + (ci * 9 + tap) * COUT + g * CO_PER + j, acc[tap][j]);
    if (ci == 0) {
#pragma unroll
        for (int j = 0; j < CO_PER; ++j) atomicAdd(db + g * CO_PER + j, bacc[j]);
    }
}

// wf[co][8 - tap][ci] = wt[ci][tap][co]
__global__ void flip_weights(const float* __restrict__ wt, float* __restrict__ wf, int cin,
                             int cout) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cin * 9 * cout) return;
    const int co = i % cout, tap = (i / cout) % 9, ci = i / (9 * cout);
    wf[(co * 9 + (8 - tap)) * cin + ci] = wt[i];
}

__global__ void relu_bwd(float* __restrict__ g, const float* __restrict__ act, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !(act[i] > 0.0f)) g[i] = 0.0f;
}

// g = 2 (y - t) / n; loss[0] += sum (y - t)^2 / n, one atomic per CTA.
__global__ void mse_grad(const float* __restrict__ y, const float* __restrict__ t,
                         float* __restrict__ g, float* __restrict__ loss, size_t n) {
    __shared__ float part[8];
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    float e = 0.0f;
    if (i < n) {
        const float d = y[i] - t[i];
        g[i] = 2.0f * d / (float)n;
        e = d * d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += part[w];
        atomicAdd(loss, s / (float)n);
    }
}

// Adam (Kingma & Ba, 2015) with bias correction factors bc1 = 1 - b1^k,
// bc2 = 1 - b2^k.
__global__ void adam_step(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps,
                          float bc1, float bc2) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// Tile mean and (std + 1) of one value per thread of a 256-thread CTA.
__device__ __forceinline__ float2 tile_scale(float dv, float* red) {
    float s1 = dv, s2 = dv * dv;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = s1;
        red[8 + (threadIdx.x >> 5)] = s2;
    }
    __syncthreads();
    float a = 0.0f, q = 0.0f;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        a += red[w];
        q += red[8 + w];
    }
    const float mu = a * (1.0f / 256.0f);
    const float sd = sqrtf(fmaxf(q * (1.0f / 256.0f) - mu * mu, 0.0f)) + 1.0f;
    return make_float2(mu, sd);
}

__global__ void __launch_bounds__(256) features(const float* __restrict__ d,
                                                const float* __restrict__ gam,
                                                float* __restrict__ x, float* __restrict__ scale,
                                                int n) {
    __shared__ float red[16];
    const int t = blockIdx.x;
    if (t >= n) return;
    const float dv = d[(size_t)t * 256 + threadIdx.x], gv = gam[(size_t)t * 256 + threadIdx.x];
    const float2 ms = tile_scale(dv, red);
    x[(size_t)t * 512 + threadIdx.x] = (dv - ms.x) / ms.y;
    x[(size_t)t * 512 + 256 + threadIdx.x] = sqrtf(fmaxf(dv, 0.0f) + fmaxf(gv, 0.0f)) / ms.y;
    if (threadIdx.x == 0) {
        scale[2 * t] = ms.x;
        scale[2 * t + 1] = ms.y;
    }
}

// ---- fused inference -------------------------------------------------------

// One conv layer from planes xin to planes yout (interior), shared memory only.
template <int CIN, int COUT, bool RELU>
__device__ __forceinline__ void layer_smem(const float* xin, float* yout, const float* wt,
                                           const float* b, int r, int c) {
    float acc[COUT];
#pragma unroll
    for (int co = 0; co < COUT; ++co) acc[co] = b[co];
    conv_pixel<CIN, COUT>(xin, wt, r, c, acc);
#pragma unroll
    for (int co = 0; co < COUT; ++co)
        yout[co * kCS + (r + 1) * kPad + c + 1] = RELU ? fmaxf(acc[co], 0.0f) : acc[co];
}

struct InferSrc {
    int tile_mode;
    const float* d;      // stack [T][H][W] or tiles [N][256]
    const float* gamma;  // [H][W] / [T][H][W] or tiles [N][256]
    long long gamma_frame_stride;
    int H, W, tiles_x, tiles_y;
    long long n_tiles;
    const StackDesc* stacks;  // batched stacks (stack mode), else null
    int n_stacks;
};

constexpr size_t infer_smem_bytes() {
    return ((size_t)round4(kParams) + 2 * (size_t)round4(kC * kCS)) * sizeof(float);
}

// Persistent grid; one tile per CTA at a time, activations ping-pong between
// two 32-channel plane sets, weights resident in shared memory.
__global__ void __launch_bounds__(256) infer(const InferSrc src, const float* __restrict__ params,
                                             float* __restrict__ u0) {
    extern __shared__ __align__(16) float sm[];
    float* wsm = sm;
    float* a0 = sm + round4(kParams);
    float* a1 = a0 + round4(kC * kCS);
    __shared__ float red[16];
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) wsm[i] = params[i];
    for (int i = threadIdx.x; i < 2 * round4(kC * kCS); i += blockDim.x) a0[i] = 0.0f;
    __syncthreads();
    const float* w1 = wsm;
    const float* b1 = w1 + 2 * 9 * kC;
    const float* w2 = b1 + kC;
    const float* b2 = w2 + kC * 9 * kC;
    const float* w3 = b2 + kC;
    const float* b3 = w3 + kC * 9 * kC;
    const float* w4 = b3 + kC;
    const float* b4 = w4 + kC * 9;
    const int p = threadIdx.x, r = p >> 4, c = p & 15;
    const long long per_frame = (long long)src.tiles_x * src.tiles_y;
    for (long long tile = blockIdx.x; tile < src.n_tiles; tile += gridDim.x) {
        float dv, gv;
        if (src.tile_mode) {
            dv = src.d[tile * 256 + p];
            gv = src.gamma[tile * 256 + p];
        } else {
            const float* sd = src.d;
            const float* sgam = src.gamma;
            long long gstride = src.gamma_frame_stride, lt = tile, pf = per_frame;
            int H = src.H, W = src.W, ty = src.tiles_y;
            if (src.stacks) {  // batched: the last stack whose first tile is <= tile
                int lo = 0, hi = src.n_stacks - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (src.stacks[mid].tile_begin <= tile) lo = mid;
                    else hi = mid - 1;
                }
                const StackDesc& st = src.stacks[lo];
                sd = st.data;
                sgam = st.gamma;
                gstride = st.gamma_frame_stride;
                lt = tile - st.tile_begin;
                H = st.H;
                W = st.W;
                ty = st.tiles_y;
                pf = (long long)st.tiles_x * st.tiles_y;
            }
            const int f = (int)(lt / pf);
            const int rem = (int)(lt - (long long)f * pf);
            const int ti = rem / ty, tj = rem - ti * ty;
            const int yy = clampi(tile_origin(ti, H) + r - 1, 0, H - 1);
            const int xx = clampi(tile_origin(tj, W) + c - 1, 0, W - 1);
            dv = sd[(long long)f * H * W + (long long)yy * W + xx];
            gv = sgam[(long long)f * gstride + (long long)yy * W + xx];
        }
        __syncthreads();  // the previous tile is done with red[] and the planes
        const float2 ms = tile_scale(dv, red);
        a1[(r + 1) * kPad + c + 1] = (dv - ms.x) / ms.y;
        a1[kCS + (r + 1) * kPad + c + 1] = sqrtf(fmaxf(dv, 0.0f) + fmaxf(gv, 0.0f)) / ms.y;
        __syncthreads();
        layer_smem<2, kC, true>(a1, a0, w1, b1, r, c);
        __syncthreads();
        layer_smem<kC, kC, true>(a0, a1, w2, b2, r, c);
        __syncthreads();
        layer_smem<kC, kC, true>(a1, a0, w3, b3, r, c);
        __syncthreads();
        float y[1] = {b4[0]};
        conv_pixel<kC, 1>(a0, w4, r, c, y);
        const float lo = kStartFrac * fmaxf(dv + gv, 1e-3f) - gv;
        u0[tile * 256 + p] = fmaxf(fmaf(ms.y, y[0], dv), lo);
    }
}

int launch_infer(const InferSrc& src, const float* params, float* u0, cudaStream_t s) {
    const size_t smem = infer_smem_bytes();
    if (cudaFuncSetAttribute(infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return NCSB_ECUDA;
    int dev = 0, sms = 1, per_sm = 1;
    if (cudaGetDevice(&dev) != cudaSuccess) return NCSB_ECUDA;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, infer, 256, smem);
    long long grid = (long long)sms * (per_sm > 0 ? per_sm : 1);
    if (grid > src.n_tiles) grid = src.n_tiles;
    infer<<<(unsigned)grid, 256, smem, s>>>(src, params, u0);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

template <int CIN, int COUT, bool RELU>
int launch_fwd(const float* x, const float* wt, const float* b, float* y, int n, cudaStream_t s) {
    const size_t smem = ((size_t)round4(CIN * kCS) + (size_t)CIN * 9 * COUT) * sizeof(float);
    if (cudaFuncSetAttribute(conv3x3_fwd<CIN, COUT, RELU>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return NCSB_ECUDA;
    conv3x3_fwd<CIN, COUT, RELU><<<n, 256, smem, s>>>(x, wt, b, y, n);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

template <int CIN, int COUT>
int launch_wgrad(const float* x, const float* dy, float* dwt, float* db, int n, cudaStream_t s) {
    const size_t smem = ((size_t)round4(CIN * kCS) + (size_t)COUT * 257) * sizeof(float);
    if (cudaFuncSetAttribute(conv3x3_wgrad<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return NCSB_ECUDA;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int grid = 2 * sms;
    if (grid > n) grid = n;
    const int per_cta = (n + grid - 1) / grid;
    grid = (n + per_cta - 1) / per_cta;
    conv3x3_wgrad<CIN, COUT><<<grid, 256, smem, s>>>(x, dy, dwt, db, n, per_cta);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

int launch_infer_batch(const float* params, const StackDesc* stacks, int n_stacks,
                       long long n_tiles, float* u0, cudaStream_t s) {
    if (n_tiles == 0) return NCSB_OK;
    InferSrc src{};
    src.tile_mode = 0;
    src.stacks = stacks;
    src.n_stacks = n_stacks;
    src.tiles_x = 1;
    src.tiles_y = 1;
    src.n_tiles = n_tiles;
    return launch_infer(src, params, u0, s);
}

}  // namespace net
}  // namespace ncsb

using namespace ncsb::net;
using ncsb::tiles_along;

extern "C" {

int ncsb_net_param_count(void) { return kParams; }

int ncsb_net_conv_fwd(const float* x, const float* wt, const float* b, float* y, int n, int cin,
                      int cout, int relu, void* stream) {
    if (!x || !wt || !y || n < 0) return NCSB_EINVAL;
    if (n == 0) return NCSB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (cin == 2 && cout == 32)
        return relu ? launch_fwd<2, 32, true>(x, wt, b, y, n, s) : launch_fwd<2, 32, false>(x, wt, b, y, n, s);
    if (cin == 32 && cout == 32)
        return relu ? launch_fwd<32, 32, true>(x, wt, b, y, n, s) : launch_fwd<32, 32, false>(x, wt, b, y, n, s);
    if (cin == 32 && cout == 1)
        return relu ? launch_fwd<32, 1, true>(x, wt, b, y, n, s) : launch_fwd<32, 1, false>(x, wt, b, y, n, s);
    if (cin == 1 && cout == 32)
        return relu ? launch_fwd<1, 32, true>(x, wt, b, y, n, s) : launch_fwd<1, 32, false>(x, wt, b, y, n, s);
    return NCSB_EINVAL;
}

int ncsb_net_conv_wgrad(const float* x, const float* dy, float* dwt, float* db, int n, int cin,
                        int cout, void* stream) {
    if (!x || !dy || !dwt || !db || n < 0) return NCSB_EINVAL;
    if (n == 0) return NCSB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (cin == 2 && cout == 32) return launch_wgrad<2, 32>(x, dy, dwt, db, n, s);
    if (cin == 32 && cout == 32) return launch_wgrad<32, 32>(x, dy, dwt, db, n, s);
    if (cin == 32 && cout == 1) return launch_wgrad<32, 1>(x, dy, dwt, db, n, s);
    return NCSB_EINVAL;
}

int ncsb_net_flip(const float* wt, float* wf, int cin, int cout, void* stream) {
    if (!wt || !wf || cin < 1 || cout < 1 || cin > 1024 || cout > 1024) return NCSB_EINVAL;
    const int n = cin * 9 * cout;
    flip_weights<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(wt, wf, cin, cout);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

int ncsb_net_relu_bwd(float* g, const float* act, int64_t n, void* stream) {
    if (!g || !act || n < 0) return NCSB_EINVAL;
    if (n == 0) return NCSB_OK;
    relu_bwd<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(g, act, (size_t)n);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

int ncsb_net_mse_grad(const float* y, const float* t, float* g, float* loss, int64_t n,
                      void* stream) {
    if (!y || !t || !g || !loss || n <= 0) return NCSB_EINVAL;
    mse_grad<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(y, t, g, loss, (size_t)n);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

int ncsb_net_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr, float b1,
                  float b2, float eps, int step, void* stream) {
    if (!w || !g || !m || !v || n < 0 || step < 1) return NCSB_EINVAL;
    if (n == 0) return NCSB_OK;
    double p1 = 1.0, p2 = 1.0;
    for (int i = 0; i < step && i < 100000; ++i) {
        p1 *= b1;
        p2 *= b2;
    }
    adam_step<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        w, g, m, v, (size_t)n, lr, b1, b2, eps, (float)(1.0 - p1), (float)(1.0 - p2));
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

int ncsb_net_features(const float* d, const float* gamma, float* x, float* scale, int n,
                      void* stream) {
    if (!d || !gamma || !x || !scale || n < 0) return NCSB_EINVAL;
    if (n == 0) return NCSB_OK;
    features<<<n, 256, 0, (cudaStream_t)stream>>>(d, gamma, x, scale, n);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

int ncsb_net_infer_stack(const float* params, const float* images, int n_frames, int height,
                         int width, const float* gamma, int gamma_per_frame, float* u0,
                         void* stream) {
    if (!params || !images || !gamma || !u0 || n_frames < 0 || height <= 0 || width <= 0)
        return NCSB_EINVAL;
    if (height < 14 || width < 14) return NCSB_ESIZE;
    if (n_frames == 0) return NCSB_OK;
    InferSrc src{};
    src.tile_mode = 0;
    src.d = images;
    src.gamma = gamma;
    src.gamma_frame_stride = gamma_per_frame ? (long long)height * width : 0;
    src.H = height;
    src.W = width;
    src.tiles_x = tiles_along(height);
    src.tiles_y = tiles_along(width);
    src.n_tiles = (long long)n_frames * src.tiles_x * src.tiles_y;
    return launch_infer(src, params, u0, (cudaStream_t)stream);
}

int ncsb_net_infer_tiles(const float* params, const float* d, const float* gamma, int64_t n_tiles,
                         float* u0, void* stream) {
    if (!params || !d || !gamma || !u0 || n_tiles < 0) return NCSB_EINVAL;
    if (n_tiles == 0) return NCSB_OK;
    InferSrc src{};
    src.tile_mode = 1;
    src.d = d;
    src.gamma = gamma;
    src.tiles_x = 1;
    src.tiles_y = 1;
    src.H = 16;
    src.W = 16;
    src.n_tiles = n_tiles;
    return launch_infer(src, params, u0, (cudaStream_t)stream);
}

}  // extern "C"
