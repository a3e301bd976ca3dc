// ncs_sim.cu -- the synthetic-data simulator on the GPU: emitters rendered
// through a pixel-integrated Gaussian PSF, then the sCMOS camera (Poisson shot
// noise, per-pixel gain, Gaussian read noise, offset).  It replaces the
// host-side loops of the reference's simulators (python3-6/pyNCS/
// denoisetools.py:118-186 genidealimage / SRhist, :205-225 addnoise /
// gendatastack) so warm-start training data can be generated at scale.
//
// Determinism: every random draw comes from a counter-based generator keyed
// by the seed and addressed by (frame, pixel, draw index), so a stack is a
// pure function of its inputs and seed regardless of launch geometry; the
// renderer sums each pixel's emitters in a fixed order (emitters sorted by
// 8 x 8-pixel cell, no atomics).
//
// Published algorithms restated here:
//   * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
//     as easy as 1, 2, 3", SC 2011): 10 rounds of two 32x32->64 multiplies
//     with the paper's multipliers and Weyl key increments;
//   * Poisson by inversion (lambda < 10) and by the transformed rejection
//     method with squeeze PTRS (W. Hormann, "The transformed rejection method
//     for generating Poisson random variables", Insurance: Mathematics and
//     Economics 12, 1993) for lambda >= 10;
//   * normal deviates by the Box-Muller transform.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "../../include/ncs_b200.h"

namespace ncsb {
namespace simk {

// ---- Philox4x32-10 ----------------------------------------------------------
struct U4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox_round(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    return U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
}

__device__ __forceinline__ U4 philox(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        c = philox_round(c, k0, k1);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// uniform in (0, 1): 24 random bits, centred in their bucket
__device__ __forceinline__ float unif(uint32_t v) {
    return ((float)(v >> 8) + 0.5f) * (1.0f / 16777216.0f);
}

// A stream of uniforms for one (frame, pixel): counter (pixel, frame, block, 0).
struct Stream {
    uint32_t k0, k1, pix, frame, block;
    int used;
    U4 buf;
    __device__ float next() {
        if (used == 4) {
            buf = philox(U4{pix, frame, block, 0u}, k0, k1);
            ++block;
            used = 0;
        }
        const uint32_t v = used == 0 ? buf.x : used == 1 ? buf.y : used == 2 ? buf.z : buf.w;
        ++used;
        return unif(v);
    }
};

// Poisson(lam).  Inversion for small means; PTRS (Hormann 1993) otherwise,
// with a bound on the rejection loop (the method accepts with probability
// above 0.9, so the bound is never the exit in practice).
__device__ int poisson(float lam, Stream& st) {
    if (!(lam > 0.0f)) return 0;
    if (lam < 10.0f) {
        const float u = st.next();
        float p = expf(-lam), F = p;
        int k = 0;
        while (u > F && k < 200) {
            ++k;
            p *= lam / (float)k;
            F += p;
        }
        return k;
    }
    const float slam = sqrtf(lam);
    const float b = 0.931f + 2.53f * slam;
    const float a = -0.059f + 0.02483f * b;
    const float invalpha = 1.1239f + 1.1328f / (b - 3.4f);
    const float vr = 0.9277f - 3.6224f / (b - 2.0f);
    for (int tries = 0; tries < 256; ++tries) {
        const float U = st.next() - 0.5f;
        const float V = st.next();
        const float us = 0.5f - fabsf(U);
        const float kf = floorf((2.0f * a / us + b) * U + lam + 0.43f);
        if (us >= 0.07f && V <= vr) return (int)kf;
        if (kf < 0.0f || (us < 0.013f && V > us)) continue;
        // the exact test cancels terms of order lam log lam: FP64
        if (log((double)V) + log((double)invalpha) - log((double)a / ((double)us * us) + b) <=
            -(double)lam + (double)kf * log((double)lam) - lgamma((double)kf + 1.0))
            return (int)kf;
    }
    return (int)floorf(lam + 0.5f);
}

__device__ __forceinline__ float normal(Stream& st) {
    const float u1 = st.next(), u2 = st.next();
    return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

// ---- rendering --------------------------------------------------------------
constexpr int kCell = 8;

// ideal[y][x] = bg + sum_e photons_e * Px_e(x) * Py_e(y) over emitters with
// |floor(x_e) - x| <= half and |floor(y_e) - y| <= half, where
// Px(x) = (erf((x + 1 - x_e) / (sqrt 2 sigma)) - erf((x - x_e) / (sqrt 2 sigma))) / 2
// (pixel x spans [x, x + 1)).  em: [n][3] (x along W, y along H, photons),
// sorted by cell; cell_start: [ncells + 1] offsets.
__global__ void render(const float* __restrict__ em, const int* __restrict__ cell_start, int ncx,
                       int ncy, int H, int W, double s2, int half, float bg,
                       float* __restrict__ ideal) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)H * W) return;
    const int y = (int)(idx / W), x = (int)(idx - (long long)y * W);
    double acc = 0.0;
    const int cy0 = max(0, (y - half) / kCell - 1), cy1 = min(ncy - 1, (y + half) / kCell + 1);
    const int cx0 = max(0, (x - half) / kCell - 1), cx1 = min(ncx - 1, (x + half) / kCell + 1);
    for (int cy = cy0; cy <= cy1; ++cy)
        for (int cx = cx0; cx <= cx1; ++cx) {
            const int c = cy * ncx + cx;
            for (int e = cell_start[c]; e < cell_start[c + 1]; ++e) {
                const double ex = em[3 * e], ey = em[3 * e + 1], ph = em[3 * e + 2];
                const int fx = (int)floor(ex), fy = (int)floor(ey);
                if (abs(fx - x) > half || abs(fy - y) > half) continue;
                const double px = 0.5 * (erf((x + 1 - ex) / s2) - erf((x - ex) / s2));
                const double py = 0.5 * (erf((y + 1 - ey) / s2) - erf((y - ey) / s2));
                acc += ph * py * px;
            }
        }
    ideal[idx] = (float)((double)bg + acc);
}

// ---- camera -----------------------------------------------------------------
// For frame t and pixel p: n ~ Poisson(ideal[p]), ADU = n gain + sqrt(var) z + offset
// (addnoise, denoisetools.py:205-211); photo-electrons d = (ADU - offset) / gain
// with d <= 0 set to 1e-6 (gendatastack, :213-225).
__global__ void camera(const float* __restrict__ ideal, int T, long long HW,
                       const float* __restrict__ offset, const float* __restrict__ gain,
                       const float* __restrict__ var, uint32_t k0, uint32_t k1,
                       float* __restrict__ adu, float* __restrict__ phot) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)T * HW) return;
    const int t = (int)(idx / HW);
    const long long p = idx - (long long)t * HW;
    Stream st{k0, k1, (uint32_t)p, (uint32_t)t, 0u, 4, U4{0u, 0u, 0u, 0u}};
    const int n = poisson(ideal[p], st);
    const float g = gain[p], off = offset[p];
    const float a = (float)n * g + sqrtf(var[p]) * normal(st) + off;
    if (adu) adu[idx] = a;
    if (phot) {
        const float d = (a - off) / g;
        phot[idx] = d <= 0.0f ? 1.0e-6f : d;
    }
}

// Uniform draws (tests of the generator): out[i] is the first deviate of the
// stream with counter (i, frame, 0, 0).
__global__ void uniforms(long long n, uint32_t frame, uint32_t k0, uint32_t k1, float* out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Stream st{k0, k1, (uint32_t)i, frame, 0u, 4, U4{0u, 0u, 0u, 0u}};
    out[i] = st.next();
}

// ---- genidealimage (denoisetools.py:150-186) --------------------------------
// Occupancy of the positions on the fine grid (x -> row), then, per output
// pixel of the R x R image, the zoom x zoom fine pixels' |'same' convolution|
// with the PSF kernel summed in a fixed order and divided by zoom (binimage,
// whose block order undoes genidealimage's transpose); zoom 1 keeps the
// transpose.  FP64 sums, so the image matches the reference's FP64 FFT
// convolution to FP32 rounding.

__global__ void occupancy_kernel(const float* __restrict__ xs, const float* __restrict__ ys, int n,
                                 int sz, float* __restrict__ fine) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float fx = floorf(xs[i]), fy = floorf(ys[i]);
    if (!(fx >= 0.0f && fx < (float)sz && fy >= 0.0f && fy < (float)sz)) return;  // also NaN
    fine[(long long)(int)fx * sz + (int)fy] = 1.0f;
}

// one block of zoom x zoom threads per output pixel (a, b)
__global__ void ideal_kernel(const float* __restrict__ fine, int R, int zoom,
                             const float* __restrict__ k, int ksz, float* __restrict__ out) {
    extern __shared__ double part[];
    const int a = blockIdx.x / R, b = blockIdx.x - (blockIdx.x / R) * R;
    const int t = threadIdx.x, i = a * zoom + t / zoom, j = b * zoom + t % zoom;
    const int sz = R * zoom, off = (ksz - 1) / 2;
    double acc = 0.0;
    for (int u = 0; u < ksz; ++u) {
        const int y = i + off - u;
        if (y < 0 || y >= sz) continue;
        for (int v = 0; v < ksz; ++v) {
            const int x = j + off - v;
            if (x < 0 || x >= sz) continue;
            const float f = fine[(long long)y * sz + x];
            if (f != 0.0f) acc += (double)k[u * ksz + v];
        }
    }
    part[t] = fabs(acc);
    __syncthreads();
    if (t == 0) {
        double sum = 0.0;
        for (int q = 0; q < zoom * zoom; ++q) sum += part[q];
        if (zoom == 1) out[(long long)b * R + a] = (float)sum;
        else out[(long long)a * R + b] = (float)(sum / zoom);
    }
}

}  // namespace simk
}  // namespace ncsb

using namespace ncsb::simk;

extern "C" {

int ncsb_sim_render(const float* emitters_sorted, const int* cell_start, int height, int width,
                    double sigma_px, int half, float background, float* ideal, void* stream) {
    if (!cell_start || !ideal || height <= 0 || width <= 0 || !(sigma_px > 0.0) || half < 0 ||
        half > 16)
        return NCSB_EINVAL;
    const int ncx = (width + kCell - 1) / kCell, ncy = (height + kCell - 1) / kCell;
    const long long n = (long long)height * width;
    render<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        emitters_sorted, cell_start, ncx, ncy, height, width, sqrt(2.0) * sigma_px, half,
        background, ideal);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

int ncsb_sim_camera(const float* ideal, int n_frames, int height, int width, const float* offset,
                    const float* gain, const float* variance, uint64_t seed, float* adu,
                    float* photo_electrons, void* stream) {
    if (!ideal || !offset || !gain || !variance || n_frames < 0 || height <= 0 || width <= 0)
        return NCSB_EINVAL;
    if (!adu && !photo_electrons) return NCSB_EINVAL;
    const long long HW = (long long)height * width;
    if (HW > 0xFFFFFFFFll) return NCSB_EINVAL;  // pixel index is one counter word
    const long long n = (long long)n_frames * HW;
    if (n == 0) return NCSB_OK;
    camera<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        ideal, n_frames, HW, offset, gain, variance, (uint32_t)seed, (uint32_t)(seed >> 32), adu,
        photo_electrons);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

int ncsb_sim_ideal_image(const float* xs, const float* ys, int n, int R, int zoom,
                         const float* kernel, int ksz, float* fine, float* out, void* stream) {
    if (n < 0 || R < 1 || zoom < 1 || zoom > 32 || ksz < 1 || !kernel || !fine || !out)
        return NCSB_EINVAL;
    if (n > 0 && (!xs || !ys)) return NCSB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    const long long sz = (long long)R * zoom;
    if (cudaMemsetAsync(fine, 0, sizeof(float) * sz * sz, s) != cudaSuccess) return NCSB_ECUDA;
    if (n > 0) ncsb::simk::occupancy_kernel<<<(n + 255) / 256, 256, 0, s>>>(xs, ys, n, (int)sz, fine);
    ncsb::simk::ideal_kernel<<<R * R, zoom * zoom, sizeof(double) * zoom * zoom, s>>>(
        fine, R, zoom, kernel, ksz, out);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

int ncsb_sim_uniforms(int64_t n, uint32_t frame, uint64_t seed, float* out, void* stream) {
    if (!out || n < 0 || n > 0xFFFFFFFFll) return NCSB_EINVAL;
    if (n == 0) return NCSB_OK;
    uniforms<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        n, frame, (uint32_t)seed, (uint32_t)(seed >> 32), out);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

}  // extern "C"
