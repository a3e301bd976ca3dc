/* oracle/ref_cuda/helper_math.h -- TEST INFRASTRUCTURE ONLY.
 *
 * The reference CUDA kernel (cuda/ncs.cu:38) includes <helper_math.h> from
 * the CUDA samples, which this image does not have.  This header supplies the
 * componentwise float4 operations that kernel uses (+, -, *, / of two
 * float4s, float4 * float and float * float4, unary -, +=, dot), written
 * here from their obvious definitions, so the kernel compiles unmodified
 * where it lies. */
#pragma once
#include <cuda_runtime.h>

inline __host__ __device__ float4 operator+(float4 a, float4 b) {
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
inline __host__ __device__ float4 operator-(float4 a, float4 b) {
    return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
inline __host__ __device__ float4 operator*(float4 a, float4 b) {
    return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w);
}
inline __host__ __device__ float4 operator/(float4 a, float4 b) {
    return make_float4(a.x / b.x, a.y / b.y, a.z / b.z, a.w / b.w);
}
inline __host__ __device__ float4 operator*(float4 a, float s) {
    return make_float4(a.x * s, a.y * s, a.z * s, a.w * s);
}
inline __host__ __device__ float4 operator*(float s, float4 a) { return a * s; }
inline __host__ __device__ float4 operator-(float4 a) { return make_float4(-a.x, -a.y, -a.z, -a.w); }
inline __host__ __device__ void operator+=(float4& a, float4 b) { a = a + b; }
inline __host__ __device__ float dot(float4 a, float4 b) {
    return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}
