// emu_runtime.cpp -- the CUDA runtime calls of the reference's host code, on
// host memory (test infrastructure: part of the reference harness, see emu.h).
// "Device" pointers are host pointers, arrays and surfaces are host buffers,
// texture objects point at EmuTexObj records, GL names map to host buffers
// registered by the harness (there is no graphics stack here).
#include "emu.h"
#include "cuda_gl_interop.h"

#include <cstdlib>
#include <map>
#include <mutex>

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;
thread_local std::vector<unsigned char> emu_dyn_smem;
std::atomic<int> emu_surface_faults{0};
std::atomic<int> emu_error_count{0};

void ref_emu_check(int code, const char *what)
{
    if (code != 0) {
        emu_error_count.fetch_add(1);
        std::fprintf(stderr, "ref_emu: %s returned %d\n", what, code);
    }
}

FILE *ref_emu_fopen(const char *, const char *) { return std::fopen("/dev/null", "w"); }

// GL objects of the harness: name -> host buffer
struct EmuGL {
    void *ptr;
    size_t bytes;
    int w, h;
};
static std::map<GLuint, EmuGL> g_gl;
static std::mutex g_gl_mu;

void ref_emu_gl_bind(GLuint name, void *ptr, size_t bytes, int w, int h)
{
    std::lock_guard<std::mutex> l(g_gl_mu);
    g_gl[name] = EmuGL{ptr, bytes, w, h};
}
bool ref_emu_gl_get(GLuint name, void **ptr, size_t *bytes, int *w, int *h)
{
    std::lock_guard<std::mutex> l(g_gl_mu);
    auto it = g_gl.find(name);
    if (it == g_gl.end()) return false;
    *ptr = it->second.ptr;
    *bytes = it->second.bytes;
    if (w) *w = it->second.w;
    if (h) *h = it->second.h;
    return true;
}

struct EmuGraphicsResource {
    GLuint name;
};
struct EmuArray {
    unsigned char *data;
    int w, h, layers;
    size_t elem;
};

extern "C" {

cudaError_t cudaMalloc(void **p, size_t n)
{
    *p = std::calloc(n ? n : 1, 1);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFree(void *p)
{
    std::free(p);
    return cudaSuccess;
}
cudaError_t cudaMemset(void *p, int v, size_t n)
{
    if (p) std::memset(p, v, n);
    return cudaSuccess;
}
cudaError_t cudaMemcpy(void *d, const void *s, size_t n, enum cudaMemcpyKind)
{
    std::memmove(d, s, n);
    return cudaSuccess;
}
cudaError_t cudaMemcpyToSymbol(const void *symbol, const void *src, size_t count, size_t offset,
                               enum cudaMemcpyKind)
{
    std::memcpy((char *)symbol + offset, src, count);
    return cudaSuccess;
}
cudaError_t cudaGetSymbolAddress(void **devPtr, const void *symbol)
{
    *devPtr = (void *)symbol;
    return cudaSuccess;
}
cudaError_t cudaCreateTextureObject(cudaTextureObject_t *t, const struct cudaResourceDesc *r,
                                    const struct cudaTextureDesc *, const struct cudaResourceViewDesc *)
{
    EmuTexObj *o = new EmuTexObj{(const unsigned char *)r->res.linear.devPtr, r->res.linear.sizeInBytes};
    *t = (cudaTextureObject_t)o;
    return cudaSuccess;
}
cudaError_t cudaDestroyTextureObject(cudaTextureObject_t t)
{
    delete (EmuTexObj *)t;
    return cudaSuccess;
}
cudaError_t cudaMalloc3DArray(cudaArray_t *a, const struct cudaChannelFormatDesc *d, struct cudaExtent e,
                              unsigned int)
{
    const size_t elem = (size_t)(d->x + d->y + d->z + d->w) / 8;
    const int layers = e.depth ? (int)e.depth : 1, h = e.height ? (int)e.height : 1;
    EmuArray *r = new EmuArray{(unsigned char *)std::calloc(elem * e.width * h * layers, 1), (int)e.width, h,
                               layers, elem};
    *a = (cudaArray_t)r;
    return cudaSuccess;
}
cudaError_t cudaMallocArray(cudaArray_t *a, const struct cudaChannelFormatDesc *d, size_t w, size_t h,
                            unsigned int)
{
    const size_t elem = (size_t)(d->x + d->y + d->z + d->w) / 8;
    EmuArray *r = new EmuArray{(unsigned char *)std::calloc(elem * w * (h ? h : 1), 1), (int)w, (int)(h ? h : 1),
                               1, elem};
    *a = (cudaArray_t)r;
    return cudaSuccess;
}
cudaError_t cudaFreeArray(cudaArray_t a)
{
    EmuArray *r = (EmuArray *)a;
    if (r) {
        std::free(r->data);
        delete r;
    }
    return cudaSuccess;
}
cudaError_t cudaCreateSurfaceObject(cudaSurfaceObject_t *s, const struct cudaResourceDesc *r)
{
    EmuArray *a = (EmuArray *)r->res.array.array;
    *s = (cudaSurfaceObject_t) new EmuSurface{a->data, a->w, a->h, a->layers, a->elem};
    return cudaSuccess;
}
cudaError_t cudaDestroySurfaceObject(cudaSurfaceObject_t s)
{
    delete (EmuSurface *)s;
    return cudaSuccess;
}
struct cudaChannelFormatDesc cudaCreateChannelDesc(int x, int y, int z, int w, enum cudaChannelFormatKind f)
{
    struct cudaChannelFormatDesc d;
    d.x = x;
    d.y = y;
    d.z = z;
    d.w = w;
    d.f = f;
    return d;
}
cudaError_t cudaThreadSynchronize(void) { return cudaSuccess; }
cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }
cudaError_t cudaGetLastError(void) { return cudaSuccess; }
cudaError_t cudaPeekAtLastError(void) { return cudaSuccess; }
const char *cudaGetErrorString(cudaError_t) { return "ref_emu"; }
cudaError_t cudaGetDevice(int *d)
{
    *d = 0;
    return cudaSuccess;
}
cudaError_t cudaDeviceGetAttribute(int *v, enum cudaDeviceAttr a, int)
{
    switch (a) {
    case cudaDevAttrMaxRegistersPerMultiprocessor: *v = 65536; break;
    case cudaDevAttrMaxRegistersPerBlock: *v = 65536; break;
    case cudaDevAttrMaxSharedMemoryPerMultiprocessor: *v = 98304; break;
    case cudaDevAttrMaxSharedMemoryPerBlock: *v = 49152; break;
    case cudaDevAttrMaxBlockDimX: *v = 1024; break;
    case cudaDevAttrMaxBlockDimY: *v = 1024; break;
    case cudaDevAttrMaxGridDimX: *v = 2147483647; break;
    case cudaDevAttrWarpSize: *v = 32; break;
    case cudaDevAttrMaxThreadsPerBlock: *v = 1024; break;
    case cudaDevAttrMultiProcessorCount: *v = 8; break;
    default: *v = 0;
    }
    return cudaSuccess;
}
cudaError_t cudaFuncSetCacheConfig(const void *, enum cudaFuncCache) { return cudaSuccess; }
cudaError_t cudaFuncSetSharedMemConfig(const void *, enum cudaSharedMemConfig) { return cudaSuccess; }
cudaError_t cudaEventCreate(cudaEvent_t *e)
{
    *e = (cudaEvent_t) new double(0.0);
    return cudaSuccess;
}
cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t)
{
#ifdef _OPENMP
    *(double *)e = omp_get_wtime();
#endif
    return cudaSuccess;
}
cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
cudaError_t cudaEventElapsedTime(float *ms, cudaEvent_t a, cudaEvent_t b)
{
    *ms = (float)((*(double *)b - *(double *)a) * 1e3);
    return cudaSuccess;
}
cudaError_t cudaEventDestroy(cudaEvent_t e)
{
    delete (double *)e;
    return cudaSuccess;
}
cudaError_t cudaGraphicsMapResources(int, cudaGraphicsResource_t *, cudaStream_t) { return cudaSuccess; }
cudaError_t cudaGraphicsUnmapResources(int, cudaGraphicsResource_t *, cudaStream_t) { return cudaSuccess; }
cudaError_t cudaGraphicsUnregisterResource(cudaGraphicsResource_t r)
{
    delete (EmuGraphicsResource *)r;
    return cudaSuccess;
}
cudaError_t cudaGraphicsResourceGetMappedPointer(void **p, size_t *n, cudaGraphicsResource_t r)
{
    int w, h;
    if (!ref_emu_gl_get(((EmuGraphicsResource *)r)->name, p, n, &w, &h)) return cudaErrorInvalidValue;
    return cudaSuccess;
}
cudaError_t cudaGraphicsSubResourceGetMappedArray(cudaArray_t *, cudaGraphicsResource_t, unsigned int,
                                                  unsigned int)
{
    return cudaSuccess;
}
}  // extern "C"

cudaError_t cudaGraphicsGLRegisterBuffer(cudaGraphicsResource **res, GLuint buffer, unsigned int)
{
    *res = (cudaGraphicsResource *)new EmuGraphicsResource{buffer};
    return cudaSuccess;
}
cudaError_t cudaGraphicsGLRegisterImage(cudaGraphicsResource **res, GLuint image, GLenum, unsigned int)
{
    *res = (cudaGraphicsResource *)new EmuGraphicsResource{image};
    return cudaSuccess;
}

// GLM's infinitePerspective evaluates tan(60 rad) in binary32; pin it to the
// correctly rounded value (what a compiler's constant folding produces) rather
// than this C runtime's tanf, which is one ulp off for this argument.
extern "C" float tanf(float x) { return (float)std::tan((double)x); }
