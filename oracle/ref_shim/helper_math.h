// helper_math.h — minimal float vector operators for compiling the reference extension
// (Dolorousrtur/CCCollisions includes NVIDIA cuda-samples' Common/helper_math.h, which is
// not available here).  Written for this project from the operator definitions: each
// operator is the component-wise IEEE operation, nothing else.  Used only by the
// reference build recipe (oracle/build_ref.py); never by the product.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

inline __host__ __device__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline __host__ __device__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline __host__ __device__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
inline __host__ __device__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
inline __host__ __device__ float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
inline __host__ __device__ float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline __host__ __device__ float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
inline __host__ __device__ float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline __host__ __device__ void operator+=(float3 &a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
inline __host__ __device__ void operator-=(float3 &a, float3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
inline __host__ __device__ void operator*=(float3 &a, float s) { a.x *= s; a.y *= s; a.z *= s; }
inline __host__ __device__ void operator/=(float3 &a, float s) { a.x /= s; a.y /= s; a.z /= s; }
inline __host__ __device__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline __host__ __device__ float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline __host__ __device__ float length(float3 v) { return sqrtf(dot(v, v)); }
inline __device__ float3 normalize(float3 v) { return v * rsqrtf(dot(v, v)); }

inline __host__ __device__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
inline __host__ __device__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
inline __host__ __device__ float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
inline __host__ __device__ float2 operator/(float2 a, float s) { return make_float2(a.x / s, a.y / s); }
inline __host__ __device__ float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
