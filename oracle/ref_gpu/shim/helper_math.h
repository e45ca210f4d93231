// Restatement (from the vector algebra, not a copy) of the subset of the CUDA
// samples' helper_math.h the reference's soft-shadow code uses, for host and
// device.  Component order: dot = ((ax*bx) + (ay*by)) + (az*bz); cross =
// (ay*bz - az*by, az*bx - ax*bz, ax*by - ay*bx); normalize = v * rsqrt(dot(v, v))
// (device rsqrtf; on the host 1 / sqrtf, the samples' host definition of
// rsqrtf).  Part of the reference GPU harness build (test infrastructure).
#pragma once
#include <cuda_runtime.h>
#include <cmath>

#define RG_HD __host__ __device__ inline

RG_HD float2 make_float2(float3 a) { return make_float2(a.x, a.y); }
RG_HD float3 make_float3(float4 a) { return make_float3(a.x, a.y, a.z); }
RG_HD float3 make_float3(float s) { return make_float3(s, s, s); }
RG_HD float4 make_float4(float3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

RG_HD float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
RG_HD float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
RG_HD float2 operator*(float2 a, float b) { return make_float2(a.x * b, a.y * b); }
RG_HD float2 operator/(float2 a, float b) { return make_float2(a.x / b, a.y / b); }
RG_HD float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
RG_HD float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
RG_HD float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
RG_HD float3 operator*(float3 a, float b) { return make_float3(a.x * b, a.y * b, a.z * b); }
RG_HD float3 operator*(float b, float3 a) { return make_float3(b * a.x, b * a.y, b * a.z); }
RG_HD float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
RG_HD float3 operator/(float3 a, float b) { return make_float3(a.x / b, a.y / b, a.z / b); }
RG_HD void operator*=(float3 &a, float b) { a.x *= b; a.y *= b; a.z *= b; }
RG_HD void operator+=(float3 &a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
RG_HD void operator-=(float3 &a, float3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
RG_HD float4 operator+(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
RG_HD float4 operator-(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
RG_HD float4 operator*(float4 a, float b) { return make_float4(a.x * b, a.y * b, a.z * b, a.w * b); }

RG_HD float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
RG_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
RG_HD float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
RG_HD float3 cross(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
RG_HD float3 normalize(float3 v)
{
#ifdef __CUDA_ARCH__
    const float invLen = rsqrtf(dot(v, v));
#else
    const float invLen = 1.0f / sqrtf(dot(v, v));
#endif
    return v * invLen;
}
RG_HD float2 fminf(float2 a, float2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
RG_HD float2 fmaxf(float2 a, float2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
RG_HD float3 fminf(float3 a, float3 b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
RG_HD float3 fmaxf(float3 a, float3 b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
