// fdzb_device.cuh -- device helpers of the FDZB pipeline.
//
// Every float operation on the parity path is spelled with the _rn intrinsics:
// the compiler never fuses them into FMA, so the kernels reproduce the
// reference's FP32 arithmetic operation for operation (its --fmad=false build)
// whatever -fmad setting this translation unit is compiled with.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "fdzb_internal.h"

namespace fdzb {

constexpr unsigned kFullWarp = 0xffffffffu;

struct f3 {
    float x, y, z;
};

__device__ __forceinline__ f3 mk3(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 ld3(const float *p) { return f3{p[0], p[1], p[2]}; }
__device__ __forceinline__ f3 sub3(f3 a, f3 b)
{
    return f3{__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)};
}
__device__ __forceinline__ f3 add3(f3 a, f3 b)
{
    return f3{__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)};
}
__device__ __forceinline__ f3 mul3(f3 a, float b)
{
    return f3{__fmul_rn(a.x, b), __fmul_rn(a.y, b), __fmul_rn(a.z, b)};
}
// ((ax*bx) + (ay*by)) + (az*bz)
__device__ __forceinline__ float dot3(f3 a, f3 b)
{
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
// (ay*bz - az*by, az*bx - ax*bz, ax*by - ay*bx)
__device__ __forceinline__ f3 cross3(f3 a, f3 b)
{
    return f3{__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
              __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
              __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}

// Light-space depth w of a point: row 3 of the column-major projection
// (K/FDprojection.inl:16-19).
__device__ __forceinline__ float light_depth(const float *M, f3 t)
{
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(M[3], t.x), __fmul_rn(M[7], t.y)),
                               __fmul_rn(M[11], t.z)),
                     __fmul_rn(M[15], 1.0f));
}

// Projected (u, v, w) of a point (K/FDprojection.inl:6-14).
__device__ __forceinline__ f3 light_project(const float *M, f3 t)
{
    f3 r;
    r.z = light_depth(M, t);
    float x = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(M[0], t.x), __fmul_rn(M[4], t.y)),
                                  __fmul_rn(M[8], t.z)),
                        __fmul_rn(M[12], 1.0f));
    r.x = __fadd_rn(__fmul_rn(__fdiv_rn(x, r.z), 0.5f), 0.5f);
    float y = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(M[1], t.x), __fmul_rn(M[5], t.y)),
                                  __fmul_rn(M[9], t.z)),
                        __fmul_rn(M[13], 1.0f));
    r.y = __fadd_rn(__fmul_rn(__fdiv_rn(y, r.z), 0.5f), 0.5f);
    return r;
}

// M * (x, y, z, 1) for a column-major 4x4 M, each component summed left to
// right (K/moveModel.inl:4-12, the reference's in-place model transform).
__device__ __forceinline__ f3 transform_point(const float *m, f3 p)
{
    const float w = 1.0f;
    return f3{__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], p.x), __fmul_rn(m[4], p.y)), __fmul_rn(m[8], p.z)),
                        __fmul_rn(m[12], w)),
              __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[1], p.x), __fmul_rn(m[5], p.y)), __fmul_rn(m[9], p.z)),
                        __fmul_rn(m[13], w)),
              __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[2], p.x), __fmul_rn(m[6], p.y)), __fmul_rn(m[10], p.z)),
                        __fmul_rn(m[14], w))};
}

// Order-preserving float <-> uint32 map, so that unsigned integer max/min
// (atomics, redux.sync) implement float max/min.  NaN is never encoded.
__device__ __forceinline__ uint32_t f2o(float f)
{
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o)
{
    uint32_t u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
    return __uint_as_float(u);
}
__host__ __device__ __forceinline__ uint32_t f2o_host(float f)
{
    union {
        float f;
        uint32_t u;
    } c;
    c.f = f;
    return (c.u & 0x80000000u) ? ~c.u : (c.u | 0x80000000u);
}

__device__ __forceinline__ uint32_t lanemask_lt()
{
    uint32_t r;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
    return r;
}

// Bounded spin budget for cross-CTA waits: a wait that exceeds it records an
// error bit and gives up, so no kernel can wait forever on a shared GPU.
constexpr unsigned kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.volatile.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ void st_volatile_u32(uint32_t *p, uint32_t v)
{
    asm volatile("st.volatile.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.volatile.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ void st_volatile_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.volatile.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Index of the frame owning global index g, given ascending bases[0..n).
__device__ __forceinline__ int frame_of(const int *bases, int n, int g)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(bases + mid) <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

}  // namespace fdzb
