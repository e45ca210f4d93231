// harness_post.cuh -- last part of the reference GPU harness translation unit
// (test infrastructure).  Host globals and host helpers of K/FourD.cu:47-226
// (the sample-texture binding creates texture objects on the CUDA arrays the
// harness registered under the GL texture names), and the extern "C" entry
// point ref_gpu_frame(): it drives the reference's own FD:: API (FS/api.cpp)
// the way 4DZB/Render/Render.cpp does -- FDinit, setters, FDaddModel,
// FDsetSampleGLTex, FDsetOutputGLBuffer, FDsetView, FDregisterGLres, then per
// frame FDsetAreaLight + FDLaunch -- times each FDLaunch with CUDA events and
// copies out the reference's buffers.
#pragma once
#include "../api.h"

#include <algorithm>
#include <vector>

// Stage wrappers (see harness_pre.cuh): event k is recorded on the default
// stream before stage k and event 5 after the last one; a stage's time is the
// span between its two events (device work and host gaps alike, as the
// reference runs them: its drivers synchronise and read counts back).
#undef lightPlaneParamCal
#undef bindSampleToBin
#undef countTriBinPairNum
#undef bindTriToBin
#undef shadowCal_perSample
constexpr int kRefGpuStages = 5;   // lightPlaneParamCal .. shadowCal_perSample
static cudaEvent_t refgpu_stage_ev[kRefGpuStages + 1];
static unsigned refgpu_stage_seen;
static void refgpu_mark(int k)
{
    if (refgpu_stage_ev[k] && cudaEventRecord(refgpu_stage_ev[k], 0) == cudaSuccess) refgpu_stage_seen |= 1u << k;
}
bool lightPlaneParamCal()
{
    refgpu_mark(0);
    const bool none = refgpu_inner_lightPlaneParamCal();
    refgpu_mark(1);
    return none;
}
void bindSampleToBin()
{
    refgpu_inner_bindSampleToBin();
    refgpu_mark(2);
}
int countTriBinPairNum()
{
    const int n = refgpu_inner_countTriBinPairNum();
    refgpu_mark(3);
    return n;
}
void bindTriToBin(int pairNum)
{
    refgpu_inner_bindTriToBin(pairNum);
    refgpu_mark(4);
}
void shadowCal_perSample()
{
    refgpu_inner_shadowCal_perSample();
    refgpu_mark(5);
}

void refgpu_gl_bind_buffer(GLuint name, void *dptr, size_t bytes);
void refgpu_gl_bind_array(GLuint name, cudaArray_t arr);
cudaArray_t refgpu_gl_array(GLuint name);
int refgpu_error_count();
void refgpu_reset_errors();
const char *refgpu_first_error();

FDStaticParams h_fdStaticParams;
FDLightPlaneParams h_fdLightPlaneParams;
float2 h_fdRectangleSubConstant;
float3 h_REF_CAL_lightPos[32 * 32];
Layered2DSurfaceManager sampleRectangleSurfManager;
std::vector<FD::FDModel> FDscene;
FD::FDResult FDresult;
bool m_enable_backfacecull = true;   // K/FourD.cu:61
float m_scenes_esp = 1e-6;           // K/FourD.cu:62
int m_viewWidth = 0, m_viewHeight = 0, m_viewWidth_LOG2UP;
int m_maxTriangleNum = 0;
int m_maxVerticesNum = 0;
int m_triangleNum = 0;
int m_verteicesNum = 0;
int m_validTriangleNum;
int m_validSampleNum;
int m_validBT_PairNum;
int m_validBinNum;
GPU_INFO my_device;
int m_maxShadowCalWarpNumPerBlock;
FD::Buffer<float4> triDataBuffer;
FD::Buffer<float4> triAABBBuffer;
FD::Buffer<struct BinRange> triBinRangeBuffer;
FD::Buffer<int> binTriStartBuffer;
FD::Buffer<int> binTriEndBuffer;
FD::Buffer<int> binTriPairBinBuffer;
FD::Buffer<int> binTriPairTriBuffer;
FD::Buffer<int> triPairNumBuffer;
FD::Buffer<int> triPairNumPrefixSumBuffer;
FD::Buffer<int> binSampleStartBuffer;
FD::Buffer<int> binSampleEndBuffer;
FD::Buffer<float> binSampleMaxZBuffer;
FD::Buffer<float4> binSampleMinRangeBuffer;
FD::Buffer<int> binSamplePairBinBuffer;
FD::Buffer<int> binSamplePairSampleBuffer;
FD::Buffer<int> isBinValidBuffer;
FD::Buffer<int> isBinValidPrefixSumBuffer;
FD::Buffer<int> validBinBuffer;
FD::Buffer<float> AABB3DReduceBuffer;
FD::Buffer<int> validBuffer;
float4 modelRectangleAABB[2];
float4 sampleRectangleAABB[2];
void *g_fdAtomics_addr;
void *g_fdCounters_addr;

namespace FDSample {
GLuint GLsamplePositionTex;
GLuint GLsampleNormalTex;
cudaGraphicsResource *positionRes;
cudaArray_t positionArray;
cudaGraphicsResource *normalRes;
cudaArray_t normalArray;
static cudaTextureObject_t positionTexObj, normalTexObj;

void setGLtexture(GLuint positionTex, GLuint normalTex)
{
    GLsamplePositionTex = positionTex;
    GLsampleNormalTex = normalTex;
}
void registerGLtexture() {}
void unregisterGLtexture() {}

// K/FourD.cu:164-182: point sampling, unnormalized coordinates.  The reference
// asks for wrap addressing, which the texture unit only applies to normalized
// coordinates; clamp is what unnormalized coordinates get (the kernels only
// read texels inside the image).
static cudaTextureObject_t make_tex(cudaArray_t a)
{
    cudaResourceDesc r;
    memset(&r, 0, sizeof(r));
    r.resType = cudaResourceTypeArray;
    r.res.array.array = a;
    cudaTextureDesc t;
    memset(&t, 0, sizeof(t));
    t.addressMode[0] = cudaAddressModeClamp;
    t.addressMode[1] = cudaAddressModeClamp;
    t.filterMode = cudaFilterModePoint;
    t.readMode = cudaReadModeElementType;
    t.normalizedCoords = 0;
    cudaTextureObject_t o = 0;
    checkCudaErrors(cudaCreateTextureObject(&o, &r, &t, NULL));
    return o;
}
void mapGLtexture()
{
    positionArray = refgpu_gl_array(GLsamplePositionTex);
    normalArray = refgpu_gl_array(GLsampleNormalTex);
    positionTexObj = make_tex(positionArray);
    normalTexObj = make_tex(normalArray);
    RefGpuTex2D p{positionTexObj}, n{normalTexObj};
    checkCudaErrors(cudaMemcpyToSymbol(samplePositionTex, &p, sizeof(p)));
    checkCudaErrors(cudaMemcpyToSymbol(sampleNormalTex, &n, sizeof(n)));
}
void unmapGLtexture()
{
    checkCudaErrors(cudaDestroyTextureObject(positionTexObj));
    checkCudaErrors(cudaDestroyTextureObject(normalTexObj));
    positionTexObj = normalTexObj = 0;
}
}  // namespace FDSample

extern "C" void inline getG_Atomic_addr()
{
    checkCudaErrors(cudaGetSymbolAddress((void **)&g_fdAtomics_addr, g_fdAtomics));
}
extern "C" void inline setStaticParams()
{
    checkCudaErrors(cudaMemcpyToSymbol(c_fdStaticParams, (void *)&h_fdStaticParams, sizeof(FDStaticParams)));
}
extern "C" void inline setDynamicParams() {}
extern "C" void inline setLightPlaneParams()
{
    checkCudaErrors(cudaMemcpyToSymbol(c_fdLightPlaneParams, &h_fdLightPlaneParams, sizeof(FDLightPlaneParams)));
}
extern "C" void inline setRectangleSubConstant()
{
    checkCudaErrors(cudaMemcpyToSymbol(c_fdRectangleSubConstant, &h_fdRectangleSubConstant, sizeof(float2)));
}
extern "C" void inline setRefLightPos()
{
    checkCudaErrors(cudaMemcpyToSymbol(c_REF_CAL_lightPos, &h_REF_CAL_lightPos, sizeof(c_REF_CAL_lightPos)));
}
// api.cpp calls these from another translation unit: emit out-of-line copies
void *refgpu_keep_inline[] = {(void *)&getG_Atomic_addr, (void *)&setStaticParams,
                              (void *)&setDynamicParams, (void *)&setLightPlaneParams,
                              (void *)&setRectangleSubConstant, (void *)&setRefLightPos};

// ---------------------------------------------------------------------------
// ref_gpu_frame: frames through the reference on the GPU.
// ---------------------------------------------------------------------------
struct RefGpuIn {
    int32_t W, H;
    const float *pos, *nrm;          // host float4[W*H]
    const float *vtx;                // host, V vertices of vstride_bytes (xyz first)
    int32_t V, vstride_bytes;
    const int32_t *idx;              // host int3[T]
    int32_t T, cull;
    float esp;
    float rightRadius, topRadius, position[3], viewDir[3], upDir[3];
    int32_t lightRes;
    int32_t warmup, reps;            // untimed and timed FDLaunch calls on the same inputs
};

struct RefGpuOut {
    float *shadow;                   // host [W*H] at y*W+x (from the last launch)
    float *launch_ms;                // host [reps]: CUDA events around each FDLaunch
    float *fdlaunch_ms;              // host [reps]: FDLaunch's own return value
    int32_t num_bins, valid_samples, valid_tris, num_pairs, view_log2up, errors;
    int64_t rows_beyond_n;           // guarded quirk events, summed over all launches
    float sub[2], lp_begin[3], lp_end[3], lp_factor[2];
    float sample_aabb[8], model_aabb[8];
    char first_error[160];
    // diagnostics: surface and texture handles, the error state after FDsetView
    // (the reference leaves cudaCreateSurfaceObject unchecked), valid triangles
    int64_t surf_handle, pos_tex_handle, view_error;
    // optional host [W*H*(N+1)] at y*W+x: per sample a written marker (1 where
    // the per-sample kernel ran, else 0) and its N light-row words, from the
    // last launch (REFGPU_MASK_DUMP)
    uint32_t *masks;
    // optional host [reps * 5]: ms of each stage driver per timed launch
    // (lightPlaneParamCal, bindSampleToBin, countTriBinPairNum, bindTriToBin,
    // shadowCal_perSample); -1 where the stage did not run
    float *stage_ms;
    int32_t bins;                    // the build's bins per side (FD_MAX_LP_GRID_SIZE)
    int32_t pad0;
    int64_t q2_events;               // pairs written beyond their triangle's count (REFGPU_Q2_MARK),
                                     // summed over all launches
};

static int refgpu_round_up(int v, int m) { return (v + m - 1) / m * m; }

extern "C" int ref_gpu_frame(const RefGpuIn *in, RefGpuOut *out)
{
    static bool inited = false;
    refgpu_reset_errors();
    if (!inited) {
        FD::FDinit();
        // the per-sample kernel needs N * 4 * 512 bytes of dynamic shared
        // memory (64 KB for N = 32), above the 48 KB default
        checkCudaErrors(cudaFuncSetAttribute((const void *)shadowCal_per_sample_kernel<U32>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 32 * 4 * 512));
        inited = true;
    }
    const int W = in->W, H = in->H, S = W * H;
    const int log2up = (int)ceilf(log2f((float)W));
    const size_t pitch = (size_t)1 << log2up;
    enum : GLuint { VBO = 11, IBO = 12, POS = 21, NRM = 22, PBO = 31 };

    // device copies of the app's GL objects
    void *dVbo = nullptr, *dIbo = nullptr, *dPbo = nullptr;
    cudaArray_t aPos = nullptr, aNrm = nullptr;
    const size_t vboBytes = (size_t)in->V * in->vstride_bytes, iboBytes = (size_t)in->T * 12;
    // the reference writes results at y << ceil(log2 W) | x (a row pitch of 2^ceil(log2 W))
    const size_t pboBytes = pitch * H * sizeof(float);
    checkCudaErrors(cudaMalloc(&dVbo, vboBytes ? vboBytes : 16));
    checkCudaErrors(cudaMalloc(&dIbo, iboBytes ? iboBytes : 16));
    checkCudaErrors(cudaMalloc(&dPbo, pboBytes));
    if (vboBytes) checkCudaErrors(cudaMemcpy(dVbo, in->vtx, vboBytes, cudaMemcpyHostToDevice));
    if (iboBytes) checkCudaErrors(cudaMemcpy(dIbo, in->idx, iboBytes, cudaMemcpyHostToDevice));
    const cudaChannelFormatDesc f4 = cudaCreateChannelDesc(32, 32, 32, 32, cudaChannelFormatKindFloat);
    checkCudaErrors(cudaMallocArray(&aPos, &f4, W, H));
    checkCudaErrors(cudaMallocArray(&aNrm, &f4, W, H));
    checkCudaErrors(cudaMemcpy2DToArray(aPos, 0, 0, in->pos, (size_t)W * 16, (size_t)W * 16, H, cudaMemcpyHostToDevice));
    checkCudaErrors(cudaMemcpy2DToArray(aNrm, 0, 0, in->nrm, (size_t)W * 16, (size_t)W * 16, H, cudaMemcpyHostToDevice));
    refgpu_gl_bind_buffer(VBO, dVbo, vboBytes);
    refgpu_gl_bind_buffer(IBO, dIbo, iboBytes);
    refgpu_gl_bind_buffer(PBO, dPbo, pboBytes);
    refgpu_gl_bind_array(POS, aPos);
    refgpu_gl_bind_array(NRM, aNrm);

    FD::FDsetBackfaceCull(in->cull != 0);
    // The app passes 2^21 (4DZB/Render/Render.cpp:181).  At least a multiple of
    // the 512-thread blocks: writeTriBinPair_kernel reads its triangle's bin
    // range before the bounds check (K/Step4_RasterizeTriangleToBin.inl:164-172).
    const int maxT = std::max(1 << 21, refgpu_round_up(std::max(in->T, 1), 512));
    const int maxV = std::max(1 << 21, std::max(in->V, 1));
    FD::FDsetSceneParams(maxT, maxV);
    FD::FDsetScenesEsp(in->esp);
    FDscene.clear();
    FD::FDaddModel(VBO, IBO, (size_t)in->vstride_bytes, "scene");
    FD::FDsetSampleGLTex(POS, NRM);
    FD::FDsetOutputGLBuffer(PBO);
    FD::FDsetView(W, H);
    out->view_error = (int64_t)cudaGetLastError();
    out->surf_handle = (int64_t)sampleRectangleSurfManager.getSurface();
    FD::FDregisterGLres();
    AreaLightDes d;
    d.rightRadius = in->rightRadius;
    d.topRadius = in->topRadius;
    d.position = glm::vec3(in->position[0], in->position[1], in->position[2]);
    d.viewDir = glm::vec3(in->viewDir[0], in->viewDir[1], in->viewDir[2]);
    d.upDir = glm::vec3(in->upDir[0], in->upDir[1], in->upDir[2]);
    d.lightResWidth = in->lightRes;
    d.lightResHeight = in->lightRes;
    m_validBT_PairNum = 0;
    m_validSampleNum = 0;
    unsigned long long zero = 0;
    checkCudaErrors(cudaMemcpyToSymbol(refgpu_rows_beyond_n, &zero, sizeof(zero)));
    checkCudaErrors(cudaMemcpyToSymbol(refgpu_q2_events, &zero, sizeof(zero)));
    // mask dump: N + 1 words per output slot of the reference's padded index
    const size_t dumpWords = (size_t)(in->lightRes + 1);
    const size_t dumpBytes = pitch * H * dumpWords * sizeof(uint32_t);
    unsigned int *dDump = nullptr;
    if (out->masks) {
        checkCudaErrors(cudaMalloc(&dDump, dumpBytes));
        checkCudaErrors(cudaMemset(dDump, 0, dumpBytes));
    }
    checkCudaErrors(cudaMemcpyToSymbol(refgpu_mask_out, &dDump, sizeof(dDump)));

    // between launches the L2 (126 MB on B200) is flushed by a 256 MB write,
    // outside the timed region, so no launch starts with the previous one's
    // inputs cached
    static void *flush = nullptr;
    const size_t flushBytes = 256ull << 20;
    if (!flush) checkCudaErrors(cudaMalloc(&flush, flushBytes));
    cudaEvent_t e0, e1;
    checkCudaErrors(cudaEventCreate(&e0));
    checkCudaErrors(cudaEventCreate(&e1));
    for (auto &ev : refgpu_stage_ev) checkCudaErrors(cudaEventCreate(&ev));
    const int total = std::max(in->warmup, 0) + std::max(in->reps, 1);
    const bool trace = getenv("REFGPU_TRACE") != nullptr;
    for (int it = 0; it < total && refgpu_error_count() == 0; ++it) {
        // FDsetAreaLight before every launch: FDLaunch divides the rectangle
        // constant by f in place (K/Step2_3_defineFDbuffer.inl:24-25)
        FD::FDsetAreaLight(d);
        if (trace)
            fprintf(stderr, "[refgpu] after FDsetAreaLight: sub %g %g RF %g %g N %d\n", h_fdRectangleSubConstant.x,
                    h_fdRectangleSubConstant.y, h_fdStaticParams.light.RectangleFactor.x,
                    h_fdStaticParams.light.RectangleFactor.y, h_fdStaticParams.light.lightResWidth);
        checkCudaErrors(cudaMemset(flush, it & 0xff, flushBytes));
        checkCudaErrors(cudaDeviceSynchronize());
        checkCudaErrors(cudaEventRecord(e0, 0));
        refgpu_stage_seen = 0;
        const float own = FD::FDLaunch();
        if (trace) {
            float a[16] = {0};
            cudaMemcpy(a, AABB3DReduceBuffer.devPtr, sizeof(a), cudaMemcpyDeviceToHost);
            fprintf(stderr,
                    "[refgpu] after FDLaunch: sub %g %g valid S %d T %d pairs %d numTris %d nv %d vsf %d W %d H %d "
                    "log2 %d lp %g %g .. %g %g err %s\n",
                    h_fdRectangleSubConstant.x, h_fdRectangleSubConstant.y, m_validSampleNum, m_validTriangleNum,
                    m_validBT_PairNum, h_fdStaticParams.numTris, h_fdStaticParams.numVertices,
                    h_fdStaticParams.vertexSizeFloat, h_fdStaticParams.viewportWidth,
                    h_fdStaticParams.viewportHeight, h_fdStaticParams.viewportWidth_LOG2_UP,
                    h_fdLightPlaneParams.begin.x, h_fdLightPlaneParams.begin.y, h_fdLightPlaneParams.end.x,
                    h_fdLightPlaneParams.end.y, cudaGetErrorName(cudaGetLastError()));
            fprintf(stderr, "[refgpu] aabb buffer:");
            for (float v : a) fprintf(stderr, " %g", v);
            fprintf(stderr, "\n");
        }
        checkCudaErrors(cudaEventRecord(e1, 0));
        checkCudaErrors(cudaEventSynchronize(e1));
        float ms = 0.f;
        checkCudaErrors(cudaEventElapsedTime(&ms, e0, e1));
        const int k = it - std::max(in->warmup, 0);
        if (k >= 0) {
            if (out->launch_ms) out->launch_ms[k] = ms;
            if (out->fdlaunch_ms) out->fdlaunch_ms[k] = own;
            if (out->stage_ms)
                for (int j = 0; j < kRefGpuStages; ++j) {
                    float v = -1.f;
                    const unsigned both = (1u << j) | (1u << (j + 1));
                    if ((refgpu_stage_seen & both) == both &&
                        cudaEventElapsedTime(&v, refgpu_stage_ev[j], refgpu_stage_ev[j + 1]) != cudaSuccess)
                        v = -1.f;
                    out->stage_ms[(size_t)k * kRefGpuStages + j] = v;
                }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (auto &ev : refgpu_stage_ev) {
        cudaEventDestroy(ev);
        ev = nullptr;
    }
    FD::FDunregisterGLres();
    unsigned long long rows = 0;
    checkCudaErrors(cudaMemcpyFromSymbol(&rows, refgpu_rows_beyond_n, sizeof(rows)));
    out->rows_beyond_n = (int64_t)rows;
    unsigned long long q2 = 0;
    checkCudaErrors(cudaMemcpyFromSymbol(&q2, refgpu_q2_events, sizeof(q2)));
    out->q2_events = (int64_t)q2;
    out->pos_tex_handle = (int64_t)FDSample::positionTexObj;

    std::vector<float> pbo(pitch * H, 0.0f);
    checkCudaErrors(cudaMemcpy(pbo.data(), dPbo, pboBytes, cudaMemcpyDeviceToHost));
    if (out->shadow)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) out->shadow[(size_t)y * W + x] = pbo[((size_t)y << log2up) | x];
    if (dDump) {
        std::vector<uint32_t> dump(pitch * H * dumpWords, 0u);
        checkCudaErrors(cudaMemcpy(dump.data(), dDump, dumpBytes, cudaMemcpyDeviceToHost));
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x)
                memcpy(out->masks + ((size_t)y * W + x) * dumpWords,
                       dump.data() + (((size_t)y << log2up) | x) * dumpWords, dumpWords * sizeof(uint32_t));
        unsigned int *none = nullptr;
        checkCudaErrors(cudaMemcpyToSymbol(refgpu_mask_out, &none, sizeof(none)));
        cudaFree(dDump);
    }
    out->sub[0] = h_fdRectangleSubConstant.x;
    out->sub[1] = h_fdRectangleSubConstant.y;
    const FDLightPlaneParams &P = h_fdLightPlaneParams;
    out->lp_begin[0] = P.begin.x; out->lp_begin[1] = P.begin.y; out->lp_begin[2] = P.begin.z;
    out->lp_end[0] = P.end.x; out->lp_end[1] = P.end.y; out->lp_end[2] = P.end.z;
    out->lp_factor[0] = P.factor.x;
    out->lp_factor[1] = P.factor.y;
    memcpy(out->sample_aabb, sampleRectangleAABB, sizeof(out->sample_aabb));
    memcpy(out->model_aabb, modelRectangleAABB, sizeof(out->model_aabb));
    out->num_bins = FD_MAX_LP_GRID_SIZE * FD_MAX_LP_GRID_SIZE;
    out->bins = FD_MAX_LP_GRID_SIZE;
    out->valid_samples = m_validSampleNum;
    out->valid_tris = m_validTriangleNum;
    out->num_pairs = m_validBT_PairNum;
    out->view_log2up = log2up;

    cudaFree(dVbo);
    cudaFree(dIbo);
    cudaFree(dPbo);
    cudaFreeArray(aPos);
    cudaFreeArray(aNrm);
    out->errors = refgpu_error_count();
    snprintf(out->first_error, sizeof(out->first_error), "%s", refgpu_first_error());
    return out->errors ? 1 : 0;
}
