// harness_pre.cuh -- first part of the reference GPU harness translation unit
// (test infrastructure).  Declares what K/FourD.cu defines, in that file's
// roles, since FourD.cu itself does not compile with CUDA 12 (its legacy
// texture references, K/FourD.cu:36-37, were removed): the __constant__
// parameter blocks and the device atomics (K/FourD.cu:26-33), and the two
// sample textures as texture OBJECTS behind the same names, read through a
// tex2D overload with the reference's sampling (point filter, unnormalized
// coordinates; K/FourD.cu:167-181).  The kernel files K/*.inl follow this file
// in the order of K/FourD.cu:230-257.
#pragma once
#include <string>
#include <thrust/device_ptr.h>
#include <thrust/reduce.h>
#include <thrust/sort.h>

#include "FourD.h"
#include "../constants.h"

// file dumps of the debug paths go to /dev/null (gl_runtime.cpp)
FILE *refgpu_fopen(const char *name, const char *mode);
#define fopen refgpu_fopen

// SaveBMP1 / BYTE of 4DZB/Util/SaveBMP.h (Windows-only), used by a debug dump
typedef unsigned char BYTE;
inline void SaveBMP1(const char *, BYTE *, int, int) {}

// Pre-Volta warp intrinsics of K/Step5_2_shadowCal.inl (the per-bin kernel,
// compiled but not launched by FDLaunch): their full-warp _sync forms.
#define __shfl_xor(v, m, w) __shfl_xor_sync(0xffffffffu, (v), (m), (w))
#define __any(p) __any_sync(0xffffffffu, (p))
#define __all(p) __all_sync(0xffffffffu, (p))
#define __ballot(p) __ballot_sync(0xffffffffu, (p))

// K/FourD.cu:17-20
__inline__ __host__ __device__ float2 make_float2(float4 a) { return make_float2(a.x, a.y); }

// globals of K/FourD.cu the kernel files use without a declaration in FourD.h
extern int m_validBinNum;
extern void *g_fdAtomics_addr;

// device-side globals of K/FourD.cu:26-37
__constant__ FDStaticParams c_fdStaticParams;
__constant__ FDLightPlaneParams c_fdLightPlaneParams;
__constant__ float2 c_fdRectangleSubConstant;
__device__ FDAtomics g_fdAtomics;
__constant__ float3 c_REF_CAL_lightPos[32 * 32];

struct RefGpuTex2D {
    cudaTextureObject_t tex;
};
__constant__ RefGpuTex2D samplePositionTex;
__constant__ RefGpuTex2D sampleNormalTex;
__device__ __forceinline__ float4 tex2D(const RefGpuTex2D &t, float x, float y) { return tex2D<float4>(t.tex, x, y); }

// Harness counter: rows >= N that the per-sample kernel's row loop would index
// (reference quirk: inverted partial row filters keep bits >= N; the build
// skips such rows instead of writing past the sample's N rows of shared memory).
__device__ unsigned long long refgpu_rows_beyond_n;
#define REFGPU_ROW_GUARD(row, rows)                       \
    if ((row) >= (rows)) {                                \
        atomicAdd(&refgpu_rows_beyond_n, 1ull);           \
        continue;                                         \
    }

// Harness counter: pairs the write kernel puts beyond its triangle's counted
// slots (reference quirk: count and write kernels test different AABBs, so the
// extra pair overwrites the next triangle's first slot, racing with it).
__device__ unsigned long long refgpu_q2_events;
#define REFGPU_Q2_MARK(cnt, tid)                                                   \
    if ((cnt) >= ((const int *)c_fdStaticParams.triBinNum)[(tid)])                \
        atomicAdd(&refgpu_q2_events, 1ull);

// Harness mask dump: after the per-sample kernel's shadow store
// (K/Step5_2_shadowCalPerSample.inl:231) the sample's final light rows, when
// the harness has set refgpu_mask_out: per sample (at the kernel's output
// index) a written marker 1 followed by its N row words, N + 1 words in all.
__device__ unsigned int *refgpu_mask_out;
#define REFGPU_MASK_DUMP(sid, m, rows)                                                  \
    if (refgpu_mask_out) {                                                              \
        unsigned int *o_ = refgpu_mask_out + (size_t)(sid) * (size_t)((rows) + 1);     \
        o_[0] = 1u;                                                                     \
        for (int r_ = 0; r_ < (rows); ++r_) o_[1 + r_] = (m)[r_ * 32];                  \
    }

// Per-stage timing: the five stage drivers FDLaunch calls (FS/api.cpp:495-552,
// declared in K/FourD.h:146-154 above this point) are defined by the kernel
// files under these names; harness_post.cuh defines the original names as
// wrappers that record a CUDA event on the default stream around each call.
#define lightPlaneParamCal refgpu_inner_lightPlaneParamCal
#define bindSampleToBin refgpu_inner_bindSampleToBin
#define countTriBinPairNum refgpu_inner_countTriBinPairNum
#define bindTriToBin refgpu_inner_bindTriToBin
#define shadowCal_perSample refgpu_inner_shadowCal_perSample
