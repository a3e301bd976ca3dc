// ncs_masks.cu -- OTF masks built on the device from optics parameters.
//
// The reference builds its 16x16 noise mask on the host with genfilter
// (python3-6/pyNCS/denoisetools.py:227-261, genkspace :96-101; matlab/
// genfilter.m:31-62): a raised-cosine high-pass of the radial spatial
// frequency whose roll-off follows from the filter type -- pureN, adjustable
// (w, h) or OTFweighted.  The synthetic workloads use one more type, 1 - the
// incoherent OTF of a circular pupil inside the cutoff 2 NA / lambda.  Here
// one CTA builds one mask in FP64: as a centred 16x16 image for callers, and/or
// directly as the solver's M^2/256 table in the spectral kernel's lane layout,
// so a batch of stacks with different optics never round-trips masks through
// the host.  genpsfparam (the reference's pupil -> PSF -> OTF) is here too.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "../../include/ncs_b200.h"

namespace ncsb {
namespace masks {

__device__ __forceinline__ int bitrev3(int i) { return ((i & 1) << 2) | (i & 2) | ((i & 4) >> 2); }

// Mask value at centred grid position (y, x), y and x in 0..15 (meshgrid of
// arange(-8, 8): X = x - 8 along columns, Y = y - 8 along rows).
__device__ double mask_value(const ncsb_optics& o, int y, int x) {
    const double X = x - 8.0, Y = y - 8.0;
    const double kr = sqrt(X * X + Y * Y) / (16.0 * o.pixel_size);
    if (o.type == NCSB_MASK_INCOHERENT) {
        const double kc = 2.0 * o.na / o.wavelength;
        if (!(kr < kc)) return 1.0;
        const double r = kr / kc;
        return 1.0 - (2.0 / CUDART_PI) * (acos(r) - r * sqrt(1.0 - r * r));
    }
    double beta, T;
    if (o.type == NCSB_MASK_PUREN) {
        beta = 0.2;
        T = (1.0 - beta) * o.wavelength / 4.0 / o.na;
    } else if (o.type == NCSB_MASK_ADJUSTABLE) {
        const double kmax = 1.0 / sqrt(2.0) / o.pixel_size;
        const double w0 = o.w * o.na / o.wavelength;
        const double a = CUDART_PI / 2.0 * (kmax / w0 - 1.0);
        beta = a / (acos(1.0 - 2.0 * o.h) + a);
        T = (1.0 - beta) / w0 / 2.0;
    } else {  // NCSB_MASK_OTFWEIGHTED
        beta = 1.0;
        T = o.wavelength / 4.0 / o.na / 1.4;
    }
    double rc = 0.5 * (1.0 + cos(CUDART_PI * T / beta * (kr - (1.0 - beta) / 2.0 / T)));
    if (kr < (1.0 - beta) / 2.0 / T) rc = 1.0;
    if (kr > (1.0 + beta) / 2.0 / T) rc = 0.0;
    return 1.0 - rc;
}

// CTA b builds mask b; thread t handles the natural-order (shifted) frequency
// (kr, kc) = (t / 16, t % 16).  centred: [n][16][16] or null; lane: the
// batch's table array with mask b going to slot[b], or null.
__global__ void __launch_bounds__(256) build_masks(const ncsb_optics* __restrict__ optics, int n,
                                                   float* __restrict__ centred,
                                                   float* __restrict__ lane,
                                                   const int* __restrict__ slot) {
    const int b = blockIdx.x;
    if (b >= n) return;
    const ncsb_optics o = optics[b];
    const int kr = threadIdx.x >> 4, kc = threadIdx.x & 15;
    // shifted[kr][kc] = centred[(kr + 8) % 16][(kc + 8) % 16]
    const double m1 = mask_value(o, (kr + 8) & 15, (kc + 8) & 15);
    if (centred) centred[(size_t)b * 256 + ((kr + 8) & 15) * 16 + ((kc + 8) & 15)] = (float)m1;
    if (lane) {
        // M^2 symmetrised over k -> -k, scaled by 1/256 (as ncsb_set_otf_mask)
        const double m2 = mask_value(o, ((16 - kr) + 8) & 15, ((16 - kc) + 8) & 15);
        const float mf1 = (float)m1, mf2 = (float)m2;
        const double v = 0.5 * ((double)mf1 * mf1 + (double)mf2 * mf2) / 256.0;
        lane[(size_t)slot[b] * 256 + (2 * kc + (kr & 1)) * 8 + bitrev3(kr >> 1)] = (float)v;
    }
}

bool valid(const ncsb_optics& o) {
    if (o.type < NCSB_MASK_OTFWEIGHTED || o.type > NCSB_MASK_INCOHERENT) return false;
    if (!(o.pixel_size > 0.0) || !(o.na > 0.0) || !(o.wavelength > 0.0)) return false;
    if (o.type == NCSB_MASK_ADJUSTABLE && !(o.w > 0.0 && o.h > 0.0 && o.h < 1.0)) return false;
    return true;
}

// Launch for n optics already in device memory (d_optics); caller validated.
cudaError_t launch_masks(const ncsb_optics* d_optics, int n, float* centred, float* lane,
                         const int* d_slot, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    build_masks<<<n, 256, 0, s>>>(d_optics, n, centred, lane, d_slot);
    return cudaGetLastError();
}

// ---- genpsfparam (denoisetools.py:103-115) ----------------------------------
// pupil = |k| on the centred grid (genkspace), 0 above NA / lambda;
// PSF = |fftshift(fft2(pupil))|^2 / its sum; OTF = |fftshift(ifft2(PSF))| / its max.
// Separable DFTs in FP64, one thread per output element (R <= 1024).

__global__ void psf_pupil(int R, double px, double fmax, double2* __restrict__ z,
                          float* __restrict__ pupil) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R * R) return;
    const int y = i / R, x = i - y * R;
    const double X = x - R / 2.0, Y = y - R / 2.0;
    double kr = sqrt(X * X + Y * Y) / (R * px);
    if (kr > fmax) kr = 0.0;
    z[i] = make_double2(kr, 0.0);
    if (pupil) pupil[i] = (float)kr;
}

// out[r][v] = sum_c in[r][c] exp(sign 2 pi i v c / R)   (rows), or the same
// along columns (cols = 1): out[u][c] = sum_r in[r][c] exp(sign 2 pi i u r / R)
__global__ void psf_dft(const double2* __restrict__ in, double2* __restrict__ out, int R,
                        double sign, int cols) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R * R) return;
    const int a = i / R, b = i - a * R;  // output (row, col)
    double re = 0.0, im = 0.0;
    for (int k = 0; k < R; ++k) {
        const double2 v = cols ? in[k * R + b] : in[a * R + k];
        const int ph = ((cols ? a : b) * k) % R;
        double sn, cs;
        sincospi(2.0 * ph / R, &sn, &cs);
        sn *= sign;
        re += v.x * cs - v.y * sn;
        im += v.x * sn + v.y * cs;
    }
    out[i] = make_double2(re, im);
}

// dst[u][v] = |src[(u - R/2) mod R][(v - R/2) mod R]|^power (fftshift), power 1 or 2
__global__ void psf_shift_abs(const double2* __restrict__ src, double2* __restrict__ dst, int R,
                              int power) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R * R) return;
    const int u = i / R, v = i - u * R, h = R / 2;
    const double2 s = src[((u - h + R) % R) * R + (v - h + R) % R];
    const double m2 = s.x * s.x + s.y * s.y;
    dst[i] = make_double2(power == 2 ? m2 : sqrt(m2), 0.0);
}

// one CTA: out = in.x / (sum or max of in.x)
__global__ void psf_normalise(const double2* __restrict__ in, int n, int by_max,
                              float* __restrict__ out) {
    __shared__ double red[1024];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        acc = by_max ? fmax(acc, in[i].x) : acc + in[i].x;
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            red[threadIdx.x] = by_max ? fmax(red[threadIdx.x], red[threadIdx.x + s])
                                      : red[threadIdx.x] + red[threadIdx.x + s];
        __syncthreads();
    }
    const double d = red[0];
    for (int i = threadIdx.x; i < n; i += blockDim.x) out[i] = (float)(in[i].x / d);
}

}  // namespace masks
}  // namespace ncsb

extern "C" {

int ncsb_genpsfparam(int R, double pixel_size, double na, double wavelength, float* psf,
                     float* pupil, float* otf, void* stream) {
    if (R < 2 || R > 1024 || !(pixel_size > 0.0) || !(na > 0.0) || !(wavelength > 0.0))
        return NCSB_EINVAL;
    if (!psf && !pupil && !otf) return NCSB_EINVAL;
    using namespace ncsb::masks;
    cudaStream_t s = (cudaStream_t)stream;
    const int n = R * R, blocks = (n + 255) / 256;
    double2 *a = nullptr, *b = nullptr;
    if (cudaMallocAsync(&a, sizeof(double2) * n, s) != cudaSuccess) return NCSB_ECUDA;
    if (cudaMallocAsync(&b, sizeof(double2) * n, s) != cudaSuccess) {
        cudaFreeAsync(a, s);
        return NCSB_ECUDA;
    }
    psf_pupil<<<blocks, 256, 0, s>>>(R, pixel_size, na / wavelength, a, pupil);
    psf_dft<<<blocks, 256, 0, s>>>(a, b, R, -1.0, 0);   // fft2: rows,
    psf_dft<<<blocks, 256, 0, s>>>(b, a, R, -1.0, 1);   //       columns
    psf_shift_abs<<<blocks, 256, 0, s>>>(a, b, R, 2);   // PSF = |fftshift(.)|^2
    if (psf) psf_normalise<<<1, 1024, 0, s>>>(b, n, 0, psf);
    if (otf) {
        psf_dft<<<blocks, 256, 0, s>>>(b, a, R, 1.0, 0);  // ifft2 (unscaled: the max
        psf_dft<<<blocks, 256, 0, s>>>(a, b, R, 1.0, 1);  // normalisation removes 1/R^2)
        psf_shift_abs<<<blocks, 256, 0, s>>>(b, a, R, 1);
        psf_normalise<<<1, 1024, 0, s>>>(a, n, 1, otf);
    }
    cudaFreeAsync(a, s);
    cudaFreeAsync(b, s);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}


int ncsb_genfilter(const ncsb_optics* optics, int n, float* masks_centred, void* stream) {
    if (!optics || !masks_centred || n < 0) return NCSB_EINVAL;
    if (n == 0) return NCSB_OK;
    for (int i = 0; i < n; ++i)
        if (!ncsb::masks::valid(optics[i])) return NCSB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    ncsb_optics* d = nullptr;
    if (cudaMallocAsync(&d, sizeof(ncsb_optics) * n, s) != cudaSuccess) return NCSB_ECUDA;
    cudaError_t e = cudaMemcpyAsync(d, optics, sizeof(ncsb_optics) * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = ncsb::masks::launch_masks(d, n, masks_centred, nullptr, nullptr, s);
    // the stream orders the free after the kernel; the host copy above is
    // synchronous for pageable memory, so `optics` may be released on return
    cudaFreeAsync(d, s);
    return e == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

}  // extern "C"
