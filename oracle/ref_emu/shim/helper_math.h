// Restatement (from the vector algebra, not a copy) of the subset of the CUDA
// samples' helper_math.h the reference's soft-shadow code uses.  Component
// order: dot = ((ax*bx) + (ay*by)) + (az*bz); cross = (ay*bz - az*by,
// az*bx - ax*bz, ax*by - ay*bx); normalize = v * (1 / sqrt(dot(v, v))) on the
// host.  Part of the reference harness build (test infrastructure).
#pragma once
#include <cuda_runtime.h>
#include <cmath>

inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }
inline int max(int a, int b) { return a > b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }
inline unsigned int max(unsigned int a, unsigned int b) { return a > b ? a : b; }
inline unsigned int min(unsigned int a, unsigned int b) { return a < b ? a : b; }
inline float max(float a, float b) { return fmaxf(a, b); }
inline float min(float a, float b) { return fminf(a, b); }
inline unsigned short max(unsigned short a, int b) { return (unsigned short)(a > b ? a : b); }
inline unsigned short min(unsigned short a, int b) { return (unsigned short)(a < b ? a : b); }

inline float2 make_float2(float3 a) { return make_float2(a.x, a.y); }
inline float3 make_float3(float4 a) { return make_float3(a.x, a.y, a.z); }
inline float3 make_float3(float s) { return make_float3(s, s, s); }
inline float4 make_float4(float3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

inline float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
inline float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
inline float2 operator*(float2 a, float b) { return make_float2(a.x * b, a.y * b); }
inline float2 operator/(float2 a, float b) { return make_float2(a.x / b, a.y / b); }
inline float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
inline float3 operator*(float3 a, float b) { return make_float3(a.x * b, a.y * b, a.z * b); }
inline float3 operator*(float b, float3 a) { return make_float3(b * a.x, b * a.y, b * a.z); }
inline float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator/(float3 a, float b) { return make_float3(a.x / b, a.y / b, a.z / b); }
inline void operator*=(float3 &a, float b) { a.x *= b; a.y *= b; a.z *= b; }
inline void operator+=(float3 &a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
inline void operator-=(float3 &a, float3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
inline float4 operator+(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline float4 operator-(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
inline float4 operator*(float4 a, float b) { return make_float4(a.x * b, a.y * b, a.z * b, a.w * b); }

inline float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline float3 cross(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float3 normalize(float3 v)
{
    float invLen = rsqrtf(dot(v, v));
    return v * invLen;
}
inline float2 fminf(float2 a, float2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
inline float2 fmaxf(float2 a, float2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
inline float3 fminf(float3 a, float3 b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
inline float3 fmaxf(float3 a, float3 b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
