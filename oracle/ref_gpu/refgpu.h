// refgpu.h -- forced first include of every translation unit of the reference's
// GPU harness (test infrastructure; oracle/ref_gpu/build_ref_gpu.py).
//
// The harness runs 4DZB's own soft-shadow sources on the GPU.  There is no
// graphics stack on the machines it runs on, so the CUDA-GL interop calls of the
// reference's host code (FS/util/OpenGLinteroperate.h, K/FourD.cu:141-191) are
// renamed here to harness functions (gl_runtime.cpp) that hand out plain device
// buffers and CUDA arrays the harness registered under the GL names.  Renaming
// (instead of defining functions with the runtime's own names) keeps the static
// CUDA runtime's real entry points untouched.
#pragma once
#define cudaGraphicsMapResources refgpu_graphics_map
#define cudaGraphicsUnmapResources refgpu_graphics_unmap
#define cudaGraphicsResourceGetMappedPointer refgpu_graphics_mapped_pointer
#define cudaGraphicsSubResourceGetMappedArray refgpu_graphics_mapped_array
#define cudaGraphicsUnregisterResource refgpu_graphics_unregister
#include <cuda_runtime.h>

// (nvcc has included cuda_runtime.h before this file: declare the renamed calls)
extern "C" {
cudaError_t cudaGraphicsMapResources(int count, cudaGraphicsResource_t *resources, cudaStream_t stream);
cudaError_t cudaGraphicsUnmapResources(int count, cudaGraphicsResource_t *resources, cudaStream_t stream);
cudaError_t cudaGraphicsResourceGetMappedPointer(void **devPtr, size_t *size, cudaGraphicsResource_t resource);
cudaError_t cudaGraphicsSubResourceGetMappedArray(cudaArray_t *array, cudaGraphicsResource_t resource,
                                                  unsigned int arrayIndex, unsigned int mipLevel);
cudaError_t cudaGraphicsUnregisterResource(cudaGraphicsResource_t resource);
}

#include <cstdint>
#include <cstdio>
#include <cstring>

// MSVC spellings of the reference: __forceinline, and the integer types of
// FS/util/Util.h:39-48
#ifndef __forceinline
#define __forceinline __forceinline__
#endif
#define __int64 long long
#define __w64
// the reference's x64 target: FS/util/Util.h:11-15 selects 64-bit pointer
// operands for its inline PTX from MSVC's _M_X64
#ifndef _M_X64
#define _M_X64 1
#endif

#ifndef __CUDACC__
// the integer min / max nvcc provides to host code (FS/api.cpp:32)
inline int max(int a, int b) { return a > b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }
#endif
