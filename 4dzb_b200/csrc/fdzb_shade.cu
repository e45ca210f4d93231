// fdzb_shade.cu -- the shading pass that consumes the shadow buffer.
//
// Reference: the app's deferred shading shader (4DZB/Resources/shader/
// phoneShading.shf:25-60), fed by the G-buffer of gatherData.shf and by the
// shadow map FDLaunch writes: per pixel, intensity = 1 - shadow; for each light
// sample, ambient + (diffuse + specular) * intensity (Phong, reflection vector
// R = 2 (L.N) N - L); the average over the light samples.  A pixel whose shadow
// value is NaN is left untouched (the shader discards it).  Plain FP32 with
// the usual CUDA math (no bit-exact claim: the GLSL original leaves normalize
// and pow to the driver).  HBM-bound for one light sample (80 B in, 16 B out
// per pixel); the light-sample loop makes it ALU-bound for many.
#include <cuda_runtime.h>

#include <string>

#include "../../include/fdzb.h"
#include "fdzb_internal.h"

namespace fdzb {
namespace {

__device__ __forceinline__ float3 f3n(float3 v)
{
    const float r = rsqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return make_float3(v.x * r, v.y * r, v.z * r);
}

__global__ void __launch_bounds__(256) k_shade(int npix, const float4 *__restrict__ g0,
                                               const float4 *__restrict__ g1, const float4 *__restrict__ g2,
                                               const float4 *__restrict__ g3, const float *__restrict__ shadow,
                                               float4 *__restrict__ out, float3 cam, float3 La, float3 Ld,
                                               float3 Ls, const float *__restrict__ lights, int nl)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        const float I = 1.0f - shadow[p];
        if (isnan(I)) continue;
        const float4 a = g0[p], b = g1[p], c = g2[p], d = g3[p];
        const float3 wp = make_float3(a.x, a.y, a.z);
        const float3 N = f3n(make_float3(b.x, b.y, b.z));
        const float3 ka = make_float3(c.x, c.y, c.z), kd = make_float3(d.x, d.y, d.z);
        const float3 ks = make_float3(a.w, b.w, c.w);
        const float shin = d.w;
        const float3 V = f3n(make_float3(cam.x - wp.x, cam.y - wp.y, cam.z - wp.z));
        const float3 amb = make_float3(La.x * ka.x, La.y * ka.y, La.z * ka.z);
        float3 acc = make_float3(0.f, 0.f, 0.f);
        for (int i = 0; i < nl; ++i) {
            const float3 lp = make_float3(__ldg(lights + 3 * i), __ldg(lights + 3 * i + 1), __ldg(lights + 3 * i + 2));
            const float3 L = f3n(make_float3(lp.x - wp.x, lp.y - wp.y, lp.z - wp.z));
            const float ldn = L.x * N.x + L.y * N.y + L.z * N.z;
            const float3 R = make_float3(2.f * ldn * N.x - L.x, 2.f * ldn * N.y - L.y, 2.f * ldn * N.z - L.z);
            const float dif = fmaxf(ldn, 0.0f);
            const float spec = powf(fmaxf(R.x * V.x + R.y * V.y + R.z * V.z, 0.0f), shin);
            acc.x += amb.x + (Ld.x * kd.x * dif + Ls.x * ks.x * spec) * I;
            acc.y += amb.y + (Ld.y * kd.y * dif + Ls.y * ks.y * spec) * I;
            acc.z += amb.z + (Ld.z * kd.z * dif + Ls.z * ks.z * spec) * I;
        }
        const float inv = 1.0f / (float)nl;
        out[p] = make_float4(acc.x * inv, acc.y * inv, acc.z * inv, 1.0f);
    }
}

}  // namespace
}  // namespace fdzb

extern "C" int fdzb_shade(const fdzb_shade_desc *d, void *stream)
{
    using namespace fdzb;
    if (!d) return set_error(FDZB_ERR_INVALID_ARG, "fdzb_shade: descriptor is NULL");
    if (d->W <= 0 || d->H <= 0 || (long long)d->W * d->H > (1ll << 30))
        return set_error(FDZB_ERR_INVALID_ARG, "fdzb_shade: bad view size");
    if (!d->d_g0 || !d->d_g1 || !d->d_g2 || !d->d_g3 || !d->d_shadow || !d->d_rgba)
        return set_error(FDZB_ERR_INVALID_ARG, "fdzb_shade: NULL buffer");
    if (d->n_light_samples < 1 || d->n_light_samples > 4096 || !d->d_light_samples)
        return set_error(FDZB_ERR_INVALID_ARG, "fdzb_shade: light samples must be 1..4096 device float3");
    for (const void *p : {(const void *)d->d_g0, (const void *)d->d_g1, (const void *)d->d_g2,
                          (const void *)d->d_g3, (const void *)d->d_rgba})
        if ((uintptr_t)p & 15) return set_error(FDZB_ERR_INVALID_ARG, "fdzb_shade: float4 buffers must be 16-byte aligned");
    const int npix = d->W * d->H;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long g = (npix + 255) / 256;
    const int grid = (int)(g > (long long)sms * 8 ? (long long)sms * 8 : (g < 1 ? 1 : g));
    k_shade<<<grid, 256, 0, (cudaStream_t)stream>>>(
        npix, (const float4 *)d->d_g0, (const float4 *)d->d_g1, (const float4 *)d->d_g2, (const float4 *)d->d_g3,
        d->d_shadow, (float4 *)d->d_rgba, make_float3(d->camera_pos[0], d->camera_pos[1], d->camera_pos[2]),
        make_float3(d->La[0], d->La[1], d->La[2]), make_float3(d->Ld[0], d->Ld[1], d->Ld[2]),
        make_float3(d->Ls[0], d->Ls[1], d->Ls[2]), d->d_light_samples, d->n_light_samples);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(FDZB_ERR_CUDA, std::string("fdzb_shade: ") + cudaGetErrorString(e));
    return FDZB_OK;
}
