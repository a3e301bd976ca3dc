// ncs_internal.cuh -- device-side building blocks shared by the NCS kernels.
//
// Tile geometry (fixed by the reference GPU path, cuda/ncs.cu:41-51): 16x16
// tiles, 256 unknowns each.  A warp group (128 threads) owns one tile; thread
// t holds the two pixels (r, c) and (r + 8, c) with r = t >> 4, c = t & 15.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

namespace ncsb {

constexpr int kTile = 16;
constexpr int kPix = 256;
constexpr int kThreads = 128;  // one warp group per tile
constexpr int kMaxM = 8;       // L-BFGS history capacity
constexpr float kFitMin = 1.0e-6f;  // FITMIN, ncs.c:169 / ncs.cu:40
constexpr float kBarrierFrac = 0.01f;  // line-search trials keep u+gamma >= 1% of its value

// Per-tile solver status, identical values to cuda/ncs.cu:61-67.
enum Status : int32_t {
    kSuccess = 0,
    kUnstarted = -1,
    kReachedMaxIters = -2,
    kIncreasingGradient = -3,
    kMinimumStep = -4,
    kReachedMaxPrecision = -5,
};

// One stack of a batched launch (device copy of ncsb_stack plus its tile
// range).  Field names match SolveArgs so kernels read either the same way.
struct StackDesc {
    const float* data;             // [T][H][W]
    const float* gamma;            // [H][W] or [T][H][W]
    float* out;                    // [T][H][W]
    long long gamma_frame_stride;  // 0 or H*W
    long long tile_begin;          // first tile of this stack in the batch's order
    int T, H, W, tiles_x, tiles_y;
    float alpha;
};

// Launch description shared by every solver form.
struct SolveArgs {
    int tile_mode;                 // 0: stack in / stack out, 1: tiles in / tiles out
    const float* data;             // stack [T][H][W] or tiles [N][256]
    const float* gamma;            // [H][W], [T][H][W] or tiles [N][256]
    const float* u0;               // optional proposed start [N][256] (tile order)
    int32_t* start;                // optional [N]: 1 = proposal rejected, solve from d
    long long gamma_frame_stride;  // stack mode: 0 (shared map) or H*W
    float* out;                    // stack [T][H][W] or tiles [N][256]
    int T, H, W;
    int tiles_x, tiles_y;          // tiles along H (slow) and W (fast)
    long long n_tiles;
    int32_t* iters;                // optional [N]
    int32_t* status;               // optional [N]
    double* cost;                  // optional [N]
    int32_t* evals;                // optional [N]: 1 + line-search trials
    unsigned long long* queue;     // work counter, zero at launch
    const float* msq;              // [256] M^2/256, natural order [kr][kc], symmetrised
    float alpha, eps, c1, min_step;
    int max_iters, m;
    // batched launch (spectral form): n_stacks descriptors sorted by
    // tile_begin, and per stack the M^2/256 table in the kernel's lane layout
    const StackDesc* stacks;
    int n_stacks;
    const float* mk_lane;          // [n_stacks][256]
    // tensor-core form: set to 1 when a tensor-core wait ran out of time
    int32_t* flag;
};

// ---- tile geometry (segmentation of ncs.c:66-113, shared by every kernel) ----
// Origin of tile i along an axis of n pixels: 14 i, the last one shifted back to
// n + 2 - 16 so that it ends at the far edge of the 1-px padded frame.
__host__ __device__ __forceinline__ int tile_origin(int i, int n) {
    const int o = 14 * i, last = n + 2 - kTile;
    return o < last ? o : last;
}

__host__ __device__ __forceinline__ int clampi(int v, int lo, int hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

// Tiles along an axis: len(range(0, n + 2, 14)) with the last origin clamped to
// n + 2 - 16 and the walk stopped there (ncs.c:71-86, :136-142).
__host__ __device__ inline int tiles_along(int n) {
    const int last = n + 2 - kTile;
    int count = 0;
    for (int b = 0;; b += 14) {
        ++count;
        if (b >= last) break;
    }
    return count;
}

__device__ __forceinline__ int bitrev4(int v) {
    return ((v & 1) << 3) | ((v & 2) << 1) | ((v & 4) >> 1) | ((v & 8) >> 3);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// Twiddles of a 16-point radix-2 transform for lane v (0..15) of a
// half-warp: stage s (span h = 8 >> s) pairs lanes v and v ^ h; both use
// W16^e with e = (v & (h-1)) << s, W16 = exp(-2 pi i / 16).
struct Twiddles {
    float2 w[4];
};

__device__ __forceinline__ Twiddles make_twiddles(int v) {
    Twiddles t;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        int h = 8 >> s;
        int e = (v & (h - 1)) << s;
        float sn, cs;
        sincospif((float)e / 8.0f, &sn, &cs);  // angle 2*pi*e/16
        t.w[s] = make_float2(cs, -sn);
    }
    return t;
}

// Forward 16-point DFT across the 16 lanes of a half-warp, one complex value
// per lane, decimation in frequency: natural-order input, output in
// bit-reversed order (lane v holds X[bitrev4(v)]).  Unnormalised.
__device__ __forceinline__ float2 fft16_fwd(float2 z, int v, const Twiddles& tw) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int h = 8 >> s;
        float2 p;
        p.x = __shfl_xor_sync(0xffffffffu, z.x, h);
        p.y = __shfl_xor_sync(0xffffffffu, z.y, h);
        const bool up = (v & h) != 0;
        const float sg = up ? -1.0f : 1.0f;
        float2 t = make_float2(fmaf(sg, z.x, p.x), fmaf(sg, z.y, p.y));
        z = up ? cmul(t, tw.w[s]) : t;
    }
    return z;
}

// Inverse of fft16_fwd up to the factor 16: bit-reversed input, natural-order
// output, decimation in time with conjugate twiddles, i.e. the unnormalised
// inverse DFT sum_k X[k] exp(+2 pi i k n / 16).
__device__ __forceinline__ float2 fft16_inv(float2 z, int v, const Twiddles& tw) {
#pragma unroll
    for (int s = 3; s >= 0; --s) {
        const int h = 8 >> s;
        float2 p;
        p.x = __shfl_xor_sync(0xffffffffu, z.x, h);
        p.y = __shfl_xor_sync(0xffffffffu, z.y, h);
        const bool up = (v & h) != 0;
        const float2 hi = up ? z : p;
        const float2 lo = up ? p : z;
        const float2 wc = make_float2(tw.w[s].x, -tw.w[s].y);
        const float2 t = cmul(hi, wc);
        const float sg = up ? -1.0f : 1.0f;
        z = make_float2(fmaf(sg, t.x, lo.x), fmaf(sg, t.y, lo.y));
    }
    return z;
}

// Block-wide (one warp group) sums.  Every thread receives bitwise the same
// result (xor butterflies are order-symmetric and the four warp partials are
// added in a fixed order), so control flow that depends on it stays uniform.
// `buf` alternates between two slots so one barrier per reduction suffices.
// `red` holds two fixed 16-double slots: every reduction, whatever its K,
// writes only its own slot, so a reduction never overwrites the slot that a
// slower thread may still be reading from the previous one.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* red, int& buf) {
    static_assert(K >= 1 && K <= 4, "slot holds 4 warps x 4 values");
#pragma unroll
    for (int k = 0; k < K; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
    double* rb = red + buf * 16;
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) rb[w * K + k] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = (rb[k] + rb[K + k]) + (rb[2 * K + k] + rb[3 * K + k]);
    buf ^= 1;
}

// Warp-wide sums of 32 values at once: on return lane v holds the sum over
// the warp of v[lane].  Each halving step exchanges half of the remaining
// vector (16, 8, 4, 2, 1 values): 31 shuffles instead of 32 x 5.
__device__ __forceinline__ float warp_transpose_sum32(float (&v)[32], int lane) {
#pragma unroll
    for (int h = 16; h >= 1; h >>= 1) {
        const bool up = (lane & h) != 0;
#pragma unroll
        for (int i = 0; i < h; ++i) {
            const float send = up ? v[i] : v[i + h];
            const float keep = up ? v[i + h] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, h);
        }
    }
    return v[0];
}

// Same for N = 8, 16 or 32 values: lane v ends with the warp total of value
// v & (N - 1) (lanes that differ only above bit log2 N are combined last).
template <int N>
__device__ __forceinline__ float warp_transpose_sum(float (&v)[N], int lane) {
    static_assert(N == 8 || N == 16 || N == 32, "8, 16 or 32 values");
#pragma unroll
    for (int h = N / 2; h >= 1; h >>= 1) {
        const bool up = (lane & h) != 0;
#pragma unroll
        for (int i = 0; i < h; ++i) {
            const float send = up ? v[i] : v[i + h];
            const float keep = up ? v[i + h] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, h);
        }
    }
#pragma unroll
    for (int o = N; o < 32; o <<= 1) v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
    return v[0];
}

__device__ __forceinline__ float block_sum_f(float v, float* red, int& buf) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    float* rb = red + buf * 4;
    if ((threadIdx.x & 31) == 0) rb[threadIdx.x >> 5] = v;
    __syncthreads();
    v = (rb[0] + rb[1]) + (rb[2] + rb[3]);
    buf ^= 1;
    return v;
}

}  // namespace ncsb
