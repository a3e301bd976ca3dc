// ncs_adu.cu -- the preprocessing prologue of ncsb_reduce_noise_adu: raw
// camera counts to photo-electrons and gamma, one pass over the stack
// (denoisetools.py:222-224 and :266, matlab/genmaps.m:29-62):
//     d = (ADU - offset) / gain, d <= 0 -> 1e-6,   gamma = var / gain^2,
// with up to 4 gain / variance map pairs, each pixel taking the pair of its
// ADU level.  IEEE FP32 subtract, divide and multiply, so the solve of its
// output equals, bit for bit, the solve of frames converted with the same
// operations anywhere else.
//
// A separate pass rather than the solver's tile gather: the gather form was
// built and measured (stack512 with the per-tile cost report on: 3.72 ms
// against 3.07 ms for this pass plus the solve) -- its extra code in the
// persistent solver's tile loop cost the hot loop more than the HBM round
// trip of d that this pass adds (about 0.08 ms on stack512).
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ncs_b200.h"

namespace ncsb {
namespace adu {

// d (and gamma) of pixel p in frame t, scalar (several map pairs, or the
// remainder of a frame whose size is not a multiple of 4)
__device__ __forceinline__ void convert_one(const float* __restrict__ adu, long long i,
                                            long long p, long long hw,
                                            const float* __restrict__ offset,
                                            const float* __restrict__ gain,
                                            const float* __restrict__ var, int n_levels,
                                            const float (&lev)[3], float* __restrict__ d,
                                            float* __restrict__ gamma_frames) {
    const float av = __ldg(adu + i);
    int lv = 0;
#pragma unroll
    for (int q = 0; q < 3; ++q) lv += (q + 1 < n_levels && av >= lev[q]) ? 1 : 0;
    const long long at = (long long)lv * hw + p;
    const float gn = __ldg(gain + at);
    const float dv = (av - __ldg(offset + p)) / gn;
    d[i] = dv <= 0.0f ? 1.0e-6f : dv;
    if (gamma_frames) gamma_frames[i] = __ldg(var + at) / (gn * gn);
}

// Grid: x over groups of 4 pixels of a frame, y over frames (y-stride for
// more than 65535 frames).  With one map pair and a frame size divisible by
// 4, 16-byte loads and stores; frame 0's threads also write the gamma map.
// gamma_frames: [T][H][W] with several pairs (gamma depends on the level),
// else null.
__global__ void __launch_bounds__(256) convert(const float* __restrict__ adu, int T, long long hw,
                                               const float* __restrict__ offset,
                                               const float* __restrict__ gain,
                                               const float* __restrict__ var, int n_levels,
                                               float l0, float l1, float l2,
                                               float* __restrict__ d,
                                               float* __restrict__ gamma_frames,
                                               float* __restrict__ gamma_map) {
    const float lev[3] = {l0, l1, l2};
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // pixel group
    const long long p0 = 4 * q;
    if (p0 >= hw) return;
    const bool vec = n_levels == 1 && (hw & 3) == 0;
    for (int t = blockIdx.y; t < T; t += gridDim.y) {
        const long long i0 = (long long)t * hw + p0;
        if (vec) {
            const float4 av = __ldg(reinterpret_cast<const float4*>(adu + i0));
            const float4 off = __ldg(reinterpret_cast<const float4*>(offset + p0));
            const float4 gn = __ldg(reinterpret_cast<const float4*>(gain + p0));
            float4 dv = make_float4((av.x - off.x) / gn.x, (av.y - off.y) / gn.y,
                                    (av.z - off.z) / gn.z, (av.w - off.w) / gn.w);
            dv.x = dv.x <= 0.0f ? 1.0e-6f : dv.x;
            dv.y = dv.y <= 0.0f ? 1.0e-6f : dv.y;
            dv.z = dv.z <= 0.0f ? 1.0e-6f : dv.z;
            dv.w = dv.w <= 0.0f ? 1.0e-6f : dv.w;
            *reinterpret_cast<float4*>(d + i0) = dv;
            if (t == 0) {
                const float4 vv = __ldg(reinterpret_cast<const float4*>(var + p0));
                *reinterpret_cast<float4*>(gamma_map + p0) =
                    make_float4(vv.x / (gn.x * gn.x), vv.y / (gn.y * gn.y), vv.z / (gn.z * gn.z),
                                vv.w / (gn.w * gn.w));
            }
        } else {
            for (long long p = p0; p < p0 + 4 && p < hw; ++p) {
                convert_one(adu, (long long)t * hw + p, p, hw, offset, gain, var, n_levels, lev,
                            d, gamma_frames);
                if (t == 0 && n_levels == 1) {
                    const float gn = __ldg(gain + p);
                    gamma_map[p] = __ldg(var + p) / (gn * gn);
                }
            }
        }
    }
}

cudaError_t launch_convert(const float* adu, int T, int H, int W, const ncsb_calibration* cal,
                           float* d, float* gamma, cudaStream_t s) {
    const long long hw = (long long)H * W;
    const long long groups = (hw + 3) / 4;
    const dim3 grid((unsigned)((groups + 255) / 256), (unsigned)(T < 65535 ? T : 65535));
    const bool multi = cal->n_levels > 1;
    // 16-byte accesses need 16-byte aligned frames: the buffers are cudaMalloc'd
    // and a frame is a multiple of 4 floats whenever the vector path runs
    convert<<<grid, 256, 0, s>>>(adu, T, hw, cal->offset, cal->gain, cal->variance,
                                 cal->n_levels, cal->levels[0], cal->levels[1], cal->levels[2],
                                 d, multi ? gamma : nullptr, multi ? nullptr : gamma);
    return cudaGetLastError();
}

}  // namespace adu
}  // namespace ncsb
