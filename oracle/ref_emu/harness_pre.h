// harness_pre.h -- first part of the reference harness translation unit (test
// infrastructure).  Declares what K/FourD.cu defines, in that file's roles,
// since FourD.cu itself cannot be compiled here (legacy texture references,
// K/FourD.cu:36-37, were removed from CUDA 12): the __constant__ parameter
// blocks, the host globals, the buffers, and the block-reduction kernel of
// K/blockAABBReduce.inl in its sequential form (emu.h).
#pragma once
#include "emu.h"

#include <string>
#include <thrust/device_ptr.h>
#include <thrust/reduce.h>
#include <thrust/sort.h>

#include "FourD.h"
#include "../constants.h"

FILE *ref_emu_fopen(const char *name, const char *mode);
#define fopen ref_emu_fopen

// SaveBMP1 / BYTE of 4DZB/Util/SaveBMP.h (Windows-only) for the debug image dump
typedef unsigned char BYTE;
inline void SaveBMP1(const char *, BYTE *, int, int) {}

// globals of K/FourD.cu the kernel files use without a declaration in FourD.h
extern int m_validBinNum;
extern void *g_fdAtomics_addr;

// device-side globals of K/FourD.cu:26-37
__constant__ FDStaticParams c_fdStaticParams;
__constant__ FDLightPlaneParams c_fdLightPlaneParams;
__constant__ float2 c_fdRectangleSubConstant;
FDAtomics g_fdAtomics;
__constant__ float3 c_REF_CAL_lightPos[32 * 32];
EmuTexRef2D samplePositionTex;
EmuTexRef2D sampleNormalTex;

// block reduction kernel of K/blockAABBReduce.inl:93-153 (min/max/sum of
// 8-float AABB records): reduced in one sequential sweep into record 0.  Min
// and max are exact under any order; the sums feed only the unused average
// extents (K/Step2_3_defineFDbuffer.inl:91-97).
enum REDUCE_TYPE { reduceMaxMinOnly, reduceXYsumOnly, reduceBoth, INVALID };
template <REDUCE_TYPE reduceType> void AABBReduce_kernel(int n)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    float *a = (float *)c_fdStaticParams.aabbTempBuffer;
    if (reduceType == reduceXYsumOnly) {
        float sx = 0.f, sy = 0.f;
        for (int i = 0; i < n; ++i) {
            sx += a[(i << 1) | 0];
            sy += a[(i << 1) | 1];
        }
        a[0] = sx;
        a[1] = sy;
        return;
    }
    float r[8] = {FD_F32_MAX, FD_F32_MAX, FD_F32_MAX, 0.f, -FD_F32_MAX, -FD_F32_MAX, -FD_F32_MAX, 0.f};
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) r[k] = fminf(r[k], a[(i << 3) | k]);
        for (int k = 4; k < 7; ++k) r[k] = fmaxf(r[k], a[(i << 3) | k]);
        if (reduceType == reduceBoth) {
            r[3] += a[(i << 3) | 3];
            r[7] += a[(i << 3) | 7];
        }
    }
    for (int k = 0; k < 8; ++k)
        if (reduceType == reduceBoth || (k != 3 && k != 7)) a[k] = r[k];
}
