// emu.h -- host execution of the reference's CUDA kernels (test infrastructure).
//
// The reference harness compiles 4DZB's own kernel and host sources for the CPU
// (oracle/ref_emu/build_ref.py) so that its outputs can be produced in this
// container and frozen as golden fixtures.  This prologue provides what the
// CUDA compiler would: execution-space keywords, the thread/block built-ins,
// the intrinsics the sources use, texture and surface stand-ins, and a launch
// emulator.  A launch runs its blocks in parallel on host threads and, inside a
// block, its threads one after the other; every active kernel of the path is
// correct under that order (their threads only read shared values written by
// lower-indexed threads of the same block).  The reference's block reduction
// (K/blockAABBReduce.inl, a warp-synchronous tree that needs lock-step warps) is
// replaced by an equivalent sequential min / max / sum into the block's slot.
#pragma once
#define THRUST_DEVICE_SYSTEM THRUST_DEVICE_SYSTEM_CPP
#include <cuda_runtime.h>
#include <helper_math.h>

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string.h>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

// execution-space and storage keywords
#undef __global__
#define __global__
#undef __shared__
#define __shared__ static thread_local
#undef __constant__
#define __constant__
#undef __launch_bounds__
#define __launch_bounds__(...)
#define __forceinline inline
#ifndef __forceinline__
#define __forceinline__ inline
#endif
// MSVC-only integer types of FS/util/Util.h:39-48
#define __int64 long long
#define __w64

// built-ins
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;
extern thread_local std::vector<unsigned char> emu_dyn_smem;
extern std::atomic<int> emu_surface_faults;

inline float2 make_float2(float4 a) { return make_float2(a.x, a.y); }   // FourD.cu:17-20 helper
inline int __popc(unsigned int a) { return __builtin_popcount(a); }
inline int __popcll(unsigned long long a) { return __builtin_popcountll(a); }
inline int __ffs(int a) { return __builtin_ffs(a); }
inline int __ffs(unsigned int a) { return __builtin_ffs((int)a); }
inline int __ffsll(long long a) { return __builtin_ffsll(a); }
inline int __ffsll(unsigned long long a) { return __builtin_ffsll((long long)a); }
inline int __umul24(int a, int b) { return (int)(((long long)(a & 0xffffff)) * (b & 0xffffff)); }
inline unsigned int __umul24(unsigned int a, unsigned int b) { return (a & 0xffffffu) * (b & 0xffffffu); }
inline void __syncthreads() {}
inline void __threadfence() {}
// warp-level intrinsics appear only in the inactive per-bin kernel
// (K/Step5_2_shadowCal.inl); they must compile, they never run here
template <class T> inline T __shfl_xor(T v, int, int = 32) { return v; }
inline int __any(int p) { return p; }
inline int __all(int p) { return p; }
inline unsigned int __ballot(int p) { return p ? 1u : 0u; }
template <class T> inline T atomicOr(T *a, T v) { return __atomic_fetch_or(a, v, __ATOMIC_RELAXED); }
template <class T> inline T atomicAnd(T *a, T v) { return __atomic_fetch_and(a, v, __ATOMIC_RELAXED); }
template <class T, class U> inline T atomicAdd(T *a, U v) { return __atomic_fetch_add(a, (T)v, __ATOMIC_RELAXED); }
template <class T> inline T atomicExch(T *a, T v) { return __atomic_exchange_n(a, v, __ATOMIC_RELAXED); }
template <class T> inline T atomicMax(T *a, T v)
{
    T o = *a;
    while (o < v && !__atomic_compare_exchange_n(a, &o, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
    return o;
}
template <class T> inline T atomicMin(T *a, T v)
{
    T o = *a;
    while (o > v && !__atomic_compare_exchange_n(a, &o, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
    return o;
}

// texture references of K/FourD.cu:36-37 (2-D float4, point sampling,
// unnormalised integer coordinates, wrap addressing)
struct EmuTexRef2D {
    const float4 *data = nullptr;
    int w = 0, h = 0;
};
inline float4 tex2D(const EmuTexRef2D &t, float x, float y)
{
    int xi = (int)floorf(x), yi = (int)floorf(y);
    xi = ((xi % t.w) + t.w) % t.w;
    yi = ((yi % t.h) + t.h) % t.h;
    return t.data[(size_t)yi * t.w + xi];
}

// texture objects over linear memory: the handle is a pointer to EmuTexObj
struct EmuTexObj {
    const unsigned char *ptr;
    size_t bytes;
};
template <class T> inline T tex1Dfetch(cudaTextureObject_t obj, int i)
{
    const EmuTexObj *o = (const EmuTexObj *)obj;
    return ((const T *)o->ptr)[i];
}

// layered surfaces: the handle is a pointer to EmuSurface
struct EmuSurface {
    unsigned char *data;
    int w, h, layers;
    size_t elem;
};
inline bool emu_surf_ok(const EmuSurface *s, int xb, int y, int layer)
{
    bool ok = s && xb >= 0 && (size_t)xb / s->elem < (size_t)s->w && y >= 0 && y < s->h && layer >= 0 &&
              layer < s->layers && xb % (int)s->elem == 0;
    if (!ok) emu_surface_faults.fetch_add(1);
    return ok;
}
template <class T>
inline void surf2DLayeredwrite(T v, cudaSurfaceObject_t so, int xb, int y, int layer,
                               cudaSurfaceBoundaryMode = cudaBoundaryModeTrap)
{
    EmuSurface *s = (EmuSurface *)so;
    if (!emu_surf_ok(s, xb, y, layer)) return;
    std::memcpy(s->data + (((size_t)layer * s->h + y) * s->w) * s->elem + xb, &v, sizeof(T));
}
template <class T>
inline T surf2DLayeredread(cudaSurfaceObject_t so, int xb, int y, int layer,
                           cudaSurfaceBoundaryMode = cudaBoundaryModeTrap)
{
    EmuSurface *s = (EmuSurface *)so;
    T v{};
    if (!emu_surf_ok(s, xb, y, layer)) return v;
    std::memcpy(&v, s->data + (((size_t)layer * s->h + y) * s->w) * s->elem + xb, sizeof(T));
    return v;
}

// C++ overloads of the runtime that cuda_runtime.h offers only under nvcc
template <class T>
inline cudaError_t cudaMemcpyToSymbol(const T &symbol, const void *src, size_t count, size_t offset = 0,
                                      enum cudaMemcpyKind kind = cudaMemcpyHostToDevice)
{
    return cudaMemcpyToSymbol((const void *)&symbol, src, count, offset, kind);
}
template <class T> inline cudaError_t cudaGetSymbolAddress(void **devPtr, const T &symbol)
{
    return cudaGetSymbolAddress(devPtr, (const void *)&symbol);
}
template <class F> inline cudaError_t cudaFuncSetSharedMemConfig(F *func, enum cudaSharedMemConfig c)
{
    return cudaFuncSetSharedMemConfig((const void *)func, c);
}
template <class F> inline cudaError_t cudaFuncSetCacheConfig(F *func, enum cudaFuncCache c)
{
    return cudaFuncSetCacheConfig((const void *)func, c);
}

// launch emulation
struct EmuCfg {
    dim3 grid, block;
    size_t smem;
};
inline EmuCfg emu_cfg(dim3 g, dim3 b, size_t smem = 0) { return EmuCfg{g, b, smem}; }

template <class F> inline void emu_launch(EmuCfg c, F &&f)
{
    const long long gx = c.grid.x, gy = c.grid.y, gz = c.grid.z;
    const long long nb = gx * gy * gz;
#pragma omp parallel for schedule(dynamic, 4)
    for (long long b = 0; b < nb; ++b) {
        blockIdx = make_uint3((unsigned)(b % gx), (unsigned)((b / gx) % gy), (unsigned)(b / (gx * gy)));
        gridDim = c.grid;
        blockDim = c.block;
        emu_dyn_smem.assign(c.smem + 16, 0);
        for (unsigned z = 0; z < c.block.z; ++z)
            for (unsigned y = 0; y < c.block.y; ++y)
                for (unsigned x = 0; x < c.block.x; ++x) {
                    threadIdx = make_uint3(x, y, z);
                    f();
                }
    }
}
template <class T> inline T *emu_extern_shared() { return (T *)emu_dyn_smem.data(); }

// Block reduction (replaces K/blockAABBReduce.inl:40-153): thread 0 of the block
// stores its value, later threads combine into the block's slot.
template <typename T> struct OperatorMin {
    T operator()(const T a, const T b) const { return min(a, b); }
};
template <typename T> struct OperatorMax {
    T operator()(const T a, const T b) const { return max(a, b); }
};
template <typename T> struct OperatorAdd {
    T operator()(const T a, const T b) const { return a + b; }
};
#define REDUCE_BLOCK_SIZE 512
template <typename T, typename Oper, size_t blockSize> inline void block_reduce(T *const odata, T mySum)
{
    Oper op;
    const unsigned t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    if (t == 0) *odata = mySum;
    else *odata = op(*odata, mySum);
}
