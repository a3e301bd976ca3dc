// oracle/ref_cuda/launch.cu -- TEST INFRASTRUCTURE ONLY: the reference CUDA
// kernel (cuda/ncs.cu, compiled unmodified where it lies) with a C entry, so
// the GPU tests can check our kernels against it and the benchmark can time
// it as the reference's own plain GPU path.
//
// Launch as cuda/pyCUDANCS/ncs.py:116-125: one block of 16 threads per 16x16
// tile, data and gamma [num_sr][16][16] FP32, the mask fftshifted (DC at
// [0][0]), out [num_sr][16][16], iterations and status [num_sr].  The kernel
// reads tile blockIdx.x only and its loops are bounded (200 iterations, step
// halving down to 1e-6 for finite positive inputs).
#include "ncs.cu"

extern "C" int ref_cuda_reduce_noise_tiles(const float* data_in, const float* gamma,
                                           const float* mask_shifted, float* data_out,
                                           int* iterations, int* status, float alpha,
                                           long long num_sr, void* stream) {
    if (num_sr <= 0) return 0;
    if (num_sr > 0x7fffffffLL) return (int)cudaErrorInvalidValue;
    ncsReduceNoise<<<(unsigned)num_sr, 16, 0, (cudaStream_t)stream>>>(
        (float4*)data_in, (float4*)gamma, (float4*)mask_shifted, (float4*)data_out, iterations,
        status, alpha);
    return (int)cudaGetLastError();
}
