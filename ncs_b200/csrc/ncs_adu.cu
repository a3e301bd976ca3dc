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
// trip of d that this pass adds (about 0.06 ms on stack512).
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ncs_b200.h"

namespace ncsb {
namespace adu {

// Raw counts as the camera stores them (FP32, or unsigned 16- or 8-bit
// integers; every integer below 2^24 converts to FP32 exactly, so an integer
// stack gives the same bits as the same counts in FP32).
__device__ __forceinline__ float load1(const float* p) { return __ldg(p); }
__device__ __forceinline__ float load1(const uint16_t* p) {
    return (float)__ldg(reinterpret_cast<const unsigned short*>(p));
}
__device__ __forceinline__ float load1(const uint8_t* p) {
    return (float)__ldg(reinterpret_cast<const unsigned char*>(p));
}
__device__ __forceinline__ float4 load4(const float* p) {
    return __ldg(reinterpret_cast<const float4*>(p));
}
__device__ __forceinline__ float4 load4(const uint16_t* p) {
    const ushort4 v = __ldg(reinterpret_cast<const ushort4*>(p));
    return make_float4((float)v.x, (float)v.y, (float)v.z, (float)v.w);
}
__device__ __forceinline__ float4 load4(const uint8_t* p) {
    const uchar4 v = __ldg(reinterpret_cast<const uchar4*>(p));
    return make_float4((float)v.x, (float)v.y, (float)v.z, (float)v.w);
}

__device__ __forceinline__ float clamp_d(float dv) { return dv <= 0.0f ? 1.0e-6f : dv; }

// Frames one thread converts: its maps are loaded once per chunk and stay in
// registers, so L2 serves each map once per kFramesPerThread frames instead
// of once per frame.
constexpr int kFramesPerThread = 8;

// Grid: x over groups of 4 pixels of a frame, y over chunks of
// kFramesPerThread frames (y-stride past 65535 chunks).  vec (set by the
// host: one map pair, a frame size divisible by 4 and every pointer aligned
// for it): 4-wide loads and 16-byte stores.  gamma_frames: [T][H][W] with
// several pairs (gamma depends on the level), else null; gamma_map: [H][W],
// written by the threads of frame 0, or null.
template <typename In>
__global__ void __launch_bounds__(256) convert(const In* __restrict__ adu, int T, long long hw,
                                               const float* __restrict__ offset,
                                               const float* __restrict__ gain,
                                               const float* __restrict__ var, int n_levels,
                                               float l0, float l1, float l2, int vec,
                                               float* __restrict__ d,
                                               float* __restrict__ gamma_frames,
                                               float* __restrict__ gamma_map) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // pixel group
    const long long p0 = 4 * q;
    if (p0 >= hw) return;
    if (vec) {
        const float4 off = __ldg(reinterpret_cast<const float4*>(offset + p0));
        const float4 gn = __ldg(reinterpret_cast<const float4*>(gain + p0));
        if (blockIdx.y == 0 && gamma_map) {
            const float4 vv = __ldg(reinterpret_cast<const float4*>(var + p0));
            *reinterpret_cast<float4*>(gamma_map + p0) =
                make_float4(vv.x / (gn.x * gn.x), vv.y / (gn.y * gn.y), vv.z / (gn.z * gn.z),
                            vv.w / (gn.w * gn.w));
        }
        for (long long t0 = (long long)blockIdx.y * kFramesPerThread; t0 < T;
             t0 += (long long)gridDim.y * kFramesPerThread) {
            const int n = T - t0 < kFramesPerThread ? (int)(T - t0) : kFramesPerThread;
#pragma unroll 4
            for (int k = 0; k < n; ++k) {
                const long long i0 = (t0 + k) * hw + p0;
                const float4 av = load4(adu + i0);
                *reinterpret_cast<float4*>(d + i0) = make_float4(
                    clamp_d((av.x - off.x) / gn.x), clamp_d((av.y - off.y) / gn.y),
                    clamp_d((av.z - off.z) / gn.z), clamp_d((av.w - off.w) / gn.w));
            }
        }
        return;
    }
    for (long long t0 = (long long)blockIdx.y * kFramesPerThread; t0 < T;
         t0 += (long long)gridDim.y * kFramesPerThread) {
        const long long t1 = T - t0 < kFramesPerThread ? T : t0 + kFramesPerThread;
        for (long long t = t0; t < t1; ++t) {
            for (long long p = p0; p < p0 + 4 && p < hw; ++p) {
                const long long i = t * hw + p;
                const float av = load1(adu + i);
                // the pair of the pixel's ADU level: level k for levels[k-1] <= ADU
                int lv = 0;
                lv += (1 < n_levels && av >= l0) ? 1 : 0;
                lv += (2 < n_levels && av >= l1) ? 1 : 0;
                lv += (3 < n_levels && av >= l2) ? 1 : 0;
                const long long at = (long long)lv * hw + p;
                const float gn = __ldg(gain + at);
                d[i] = clamp_d((av - __ldg(offset + p)) / gn);
                if (gamma_frames) gamma_frames[i] = __ldg(var + at) / (gn * gn);
                if (t == 0 && gamma_map) gamma_map[p] = __ldg(var + p) / (gn * gn);
            }
        }
    }
}

// gamma = var / gain^2 of a single map pair, for callers that convert the
// stack in several launches
__global__ void __launch_bounds__(256) gamma_of(long long hw, const float* __restrict__ gain,
                                                const float* __restrict__ var,
                                                float* __restrict__ gamma) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < hw;
         p += (long long)gridDim.x * blockDim.x) {
        const float gn = __ldg(gain + p);
        gamma[p] = __ldg(var + p) / (gn * gn);
    }
}

inline bool aligned(const void* p, size_t a) { return p == nullptr || (uintptr_t)p % a == 0; }

template <typename In>
cudaError_t launch_typed(const In* adu, int T, long long hw, const ncsb_calibration* cal,
                         float* d, float* gamma_frames, float* gamma_map, cudaStream_t s) {
    const bool vec = cal->n_levels == 1 && hw % 4 == 0 && aligned(adu, 4 * sizeof(In)) &&
                     aligned(cal->offset, 16) && aligned(cal->gain, 16) &&
                     aligned(cal->variance, 16) && aligned(d, 16) && aligned(gamma_map, 16);
    const long long groups = (hw + 3) / 4;
    const long long chunks = (T + kFramesPerThread - 1) / kFramesPerThread;
    const dim3 grid((unsigned)((groups + 255) / 256), (unsigned)(chunks < 65535 ? chunks : 65535));
    convert<In><<<grid, 256, 0, s>>>(adu, T, hw, cal->offset, cal->gain, cal->variance,
                                     cal->n_levels, cal->levels[0], cal->levels[1],
                                     cal->levels[2], vec ? 1 : 0, d, gamma_frames, gamma_map);
    return cudaGetLastError();
}

// T >= 1 frames of type adu_type (NCSB_ADU_*) to d [T][H][W]; gamma_frames
// [T][H][W] (several pairs) and gamma_map [H][W] (one pair) may each be null.
cudaError_t launch_convert(const void* adu, int adu_type, int T, int H, int W,
                           const ncsb_calibration* cal, float* d, float* gamma_frames,
                           float* gamma_map, cudaStream_t s) {
    const long long hw = (long long)H * W;
    switch (adu_type) {
        case NCSB_ADU_F32:
            return launch_typed((const float*)adu, T, hw, cal, d, gamma_frames, gamma_map, s);
        case NCSB_ADU_U16:
            return launch_typed((const uint16_t*)adu, T, hw, cal, d, gamma_frames, gamma_map, s);
        case NCSB_ADU_U8:
            return launch_typed((const uint8_t*)adu, T, hw, cal, d, gamma_frames, gamma_map, s);
        default:
            return cudaErrorInvalidValue;
    }
}

cudaError_t launch_gamma_map(const ncsb_calibration* cal, long long hw, float* gamma,
                             cudaStream_t s, int num_sms) {
    long long blocks = (hw + 255) / 256;
    if (blocks > 8LL * num_sms) blocks = 8LL * num_sms;
    gamma_of<<<(unsigned)blocks, 256, 0, s>>>(hw, cal->gain, cal->variance, gamma);
    return cudaGetLastError();
}

}  // namespace adu
}  // namespace ncsb
