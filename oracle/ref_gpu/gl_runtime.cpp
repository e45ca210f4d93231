// gl_runtime.cpp -- host side of the reference GPU harness (test
// infrastructure): the GL-name registry that stands in for CUDA-GL interop
// (plain device buffers and CUDA arrays registered by ref_gpu_frame), the
// renamed interop calls of refgpu.h / shim/cuda_gl_interop.h, the error
// recorder behind checkCudaErrors, and the /dev/null target of the debug dumps.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "cuda_gl_interop.h"

namespace {
struct GLObject {
    void *dptr = nullptr;
    size_t bytes = 0;
    cudaArray_t array = nullptr;
};
struct Resource {
    GLuint name;
};
std::map<GLuint, GLObject> g_objects;
std::mutex g_mu;
int g_errors = 0;
std::string g_first;
}  // namespace

void refgpu_check(int code, const char *what, const char *file, int line)
{
    if (code == 0) return;
    std::lock_guard<std::mutex> l(g_mu);
    if (g_errors++ == 0) {
        char b[160];
        snprintf(b, sizeof(b), "%s:%d %s -> %d (%s)", file ? strrchr(file, '/') ? strrchr(file, '/') + 1 : file : "",
                 line, what, code, cudaGetErrorName((cudaError_t)code));
        g_first = b;
    }
}
int refgpu_error_count()
{
    std::lock_guard<std::mutex> l(g_mu);
    return g_errors;
}
void refgpu_reset_errors()
{
    std::lock_guard<std::mutex> l(g_mu);
    g_errors = 0;
    g_first.clear();
}
const char *refgpu_first_error() { return g_first.c_str(); }

FILE *refgpu_fopen(const char *, const char *) { return std::fopen("/dev/null", "w"); }

void refgpu_gl_bind_buffer(GLuint name, void *dptr, size_t bytes)
{
    std::lock_guard<std::mutex> l(g_mu);
    GLObject &o = g_objects[name];
    o.dptr = dptr;
    o.bytes = bytes;
    o.array = nullptr;
}
void refgpu_gl_bind_array(GLuint name, cudaArray_t arr)
{
    std::lock_guard<std::mutex> l(g_mu);
    GLObject &o = g_objects[name];
    o.dptr = nullptr;
    o.bytes = 0;
    o.array = arr;
}
cudaArray_t refgpu_gl_array(GLuint name)
{
    std::lock_guard<std::mutex> l(g_mu);
    auto it = g_objects.find(name);
    return it == g_objects.end() ? nullptr : it->second.array;
}

cudaError_t cudaGraphicsGLRegisterBuffer(cudaGraphicsResource **res, GLuint buffer, unsigned int)
{
    *res = (cudaGraphicsResource *)new Resource{buffer};
    return cudaSuccess;
}
cudaError_t cudaGraphicsGLRegisterImage(cudaGraphicsResource **res, GLuint image, GLenum, unsigned int)
{
    *res = (cudaGraphicsResource *)new Resource{image};
    return cudaSuccess;
}

extern "C" {
cudaError_t cudaGraphicsMapResources(int, cudaGraphicsResource_t *, cudaStream_t) { return cudaSuccess; }
cudaError_t cudaGraphicsUnmapResources(int, cudaGraphicsResource_t *, cudaStream_t) { return cudaSuccess; }
cudaError_t cudaGraphicsUnregisterResource(cudaGraphicsResource_t r)
{
    delete (Resource *)r;
    return cudaSuccess;
}
cudaError_t cudaGraphicsResourceGetMappedPointer(void **p, size_t *n, cudaGraphicsResource_t r)
{
    std::lock_guard<std::mutex> l(g_mu);
    auto it = g_objects.find(((Resource *)r)->name);
    if (it == g_objects.end() || !it->second.dptr) return cudaErrorInvalidValue;
    *p = it->second.dptr;
    *n = it->second.bytes;
    return cudaSuccess;
}
cudaError_t cudaGraphicsSubResourceGetMappedArray(cudaArray_t *a, cudaGraphicsResource_t r, unsigned int, unsigned int)
{
    std::lock_guard<std::mutex> l(g_mu);
    auto it = g_objects.find(((Resource *)r)->name);
    if (it == g_objects.end() || !it->second.array) return cudaErrorInvalidValue;
    *a = it->second.array;
    return cudaSuccess;
}

// GLM's infinitePerspective evaluates tan(60 rad) in binary32 on the host; pin
// it to the correctly rounded value (what a compiler's constant folding
// produces) rather than this C runtime's tanf, which is one ulp off for this
// argument.
float tanf(float x) { return (float)std::tan((double)x); }
}  // extern "C"
