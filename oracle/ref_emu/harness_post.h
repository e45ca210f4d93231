// harness_post.h -- last part of the reference harness translation unit (test
// infrastructure).  Host globals and host helpers of K/FourD.cu:47-226 (the
// sample-texture binding now points the emulated texture references at host
// images), and the extern "C" entry point ref_frame(): it drives the reference's
// own FD:: API (FS/api.cpp) the way 4DZB/Render/Render.cpp does -- FDinit,
// setters, FDaddModel, FDsetSampleGLTex, FDsetOutputGLBuffer, FDsetView,
// FDregisterGLres, FDsetAreaLight, FDLaunch -- and copies out the reference's
// buffers.
#pragma once
#include "../api.h"

void ref_emu_gl_bind(GLuint name, void *ptr, size_t bytes, int w, int h);
bool ref_emu_gl_get(GLuint name, void **ptr, size_t *bytes, int *w, int *h);
extern std::atomic<int> emu_error_count;

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
void setGLtexture(GLuint positionTex, GLuint normalTex)
{
    GLsamplePositionTex = positionTex;
    GLsampleNormalTex = normalTex;
}
void registerGLtexture() {}
void unregisterGLtexture() {}
void mapGLtexture()
{
    void *p;
    size_t n;
    int w, h;
    if (ref_emu_gl_get(GLsamplePositionTex, &p, &n, &w, &h)) samplePositionTex = EmuTexRef2D{(const float4 *)p, w, h};
    if (ref_emu_gl_get(GLsampleNormalTex, &p, &n, &w, &h)) sampleNormalTex = EmuTexRef2D{(const float4 *)p, w, h};
}
void unmapGLtexture() {}
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
void *ref_emu_keep_inline[] = {(void *)&getG_Atomic_addr, (void *)&setStaticParams,
                               (void *)&setDynamicParams, (void *)&setLightPlaneParams,
                               (void *)&setRectangleSubConstant, (void *)&setRefLightPos};

// ---------------------------------------------------------------------------
// ref_frame: one frame through the reference.
// ---------------------------------------------------------------------------
struct RefIn {
    int32_t W, H;
    const float *pos, *nrm;          // float4[W*H]
    const float *vtx;                // V vertices of vstride_bytes (xyz first)
    int32_t V, vstride_bytes;
    const int32_t *idx;              // int3[T]
    int32_t T, cull;
    float esp;
    float rightRadius, topRadius, position[3], viewDir[3], upDir[3];
    int32_t lightRes;
    int32_t nthreads;
};

struct RefOut {
    float *shadow;                   // [W*H] at y*W+x
    int32_t *sorted_keys, *sorted_vals;          // [W*H]
    int32_t *bin_sample_start, *bin_sample_end;  // [NB+1]
    float *bin_maxz, *bin_range;                 // [NB], [4*NB]
    float *tri_aabb;                             // [8*T]
    int32_t *tri_count, *tri_prefix;             // [T]
    int32_t pair_capacity;
    int32_t *sorted_pair_bin, *sorted_pair_tri;  // [pair_capacity]
    int32_t *bin_tri_start, *bin_tri_end;        // [NB]
    // scalars
    int32_t num_bins, valid_samples, valid_tris, num_pairs, view_log2up, errors;
    float ms;
    float mat[16], RF[2], corners[12], deltas[6];
    float sub[2], lp_begin[3], lp_end[3], lp_factor[2];
    float sample_aabb[8], model_aabb[8];
};

extern "C" int ref_frame(const RefIn *in, RefOut *out)
{
#ifdef _OPENMP
    if (in->nthreads > 0) omp_set_num_threads(in->nthreads);
#endif
    static bool inited = false;
    if (!inited) {
        FD::FDinit();
        inited = true;
    }
    emu_error_count.store(0);
    emu_surface_faults.store(0);
    const int W = in->W, H = in->H, S = W * H;
    const int log2up = (int)ceilf(log2f((float)W));
    const size_t pitch = (size_t)1 << log2up;
    // the reference writes results at y << ceil(log2 W) | x
    std::vector<float> pbo(pitch * H, 0.0f);
    std::vector<float4> posImg((size_t)S), nrmImg((size_t)S);
    std::memcpy(posImg.data(), in->pos, sizeof(float4) * S);
    std::memcpy(nrmImg.data(), in->nrm, sizeof(float4) * S);
    std::vector<float> vbo((size_t)in->V * in->vstride_bytes / 4);
    std::memcpy(vbo.data(), in->vtx, vbo.size() * 4);
    std::vector<int32_t> ibo((size_t)in->T * 3);
    std::memcpy(ibo.data(), in->idx, ibo.size() * 4);
    enum : GLuint { VBO = 11, IBO = 12, POS = 21, NRM = 22, PBO = 31 };
    ref_emu_gl_bind(VBO, vbo.data(), vbo.size() * 4, 0, 0);
    ref_emu_gl_bind(IBO, ibo.data(), ibo.size() * 4, 0, 0);
    ref_emu_gl_bind(POS, posImg.data(), posImg.size() * sizeof(float4), W, H);
    ref_emu_gl_bind(NRM, nrmImg.data(), nrmImg.size() * sizeof(float4), W, H);
    ref_emu_gl_bind(PBO, pbo.data(), pbo.size() * 4, 0, 0);

    FD::FDsetBackfaceCull(in->cull != 0);
    FD::FDsetSceneParams(in->T > 0 ? in->T : 1, in->V > 0 ? in->V : 1);
    FD::FDsetScenesEsp(in->esp);
    FDscene.clear();
    FD::FDaddModel(VBO, IBO, (size_t)in->vstride_bytes, "scene");
    FD::FDsetSampleGLTex(POS, NRM);
    FD::FDsetOutputGLBuffer(PBO);
    FD::FDsetView(W, H);
    FD::FDregisterGLres();
    AreaLightDes d;
    d.rightRadius = in->rightRadius;
    d.topRadius = in->topRadius;
    d.position = glm::vec3(in->position[0], in->position[1], in->position[2]);
    d.viewDir = glm::vec3(in->viewDir[0], in->viewDir[1], in->viewDir[2]);
    d.upDir = glm::vec3(in->upDir[0], in->upDir[1], in->upDir[2]);
    d.lightResWidth = in->lightRes;
    d.lightResHeight = in->lightRes;
    // clear state a previous frame could leave in buffers read before written
    m_validBT_PairNum = 0;
    m_validSampleNum = 0;
    FD::FDsetAreaLight(d);
    out->ms = FD::FDLaunch();
    FD::FDunregisterGLres();

    const AreaLight &L = h_fdStaticParams.light;
    std::memcpy(out->mat, L.upRightMat, sizeof(out->mat));
    out->RF[0] = L.RectangleFactor.x;
    out->RF[1] = L.RectangleFactor.y;
    const float3 c[4] = {L.upRightCornerPosition, L.upLeftCornerPosition, L.downLeftCornerPosition,
                         L.downRightCornerPosition};
    for (int i = 0; i < 4; ++i) {
        out->corners[3 * i] = c[i].x;
        out->corners[3 * i + 1] = c[i].y;
        out->corners[3 * i + 2] = c[i].z;
    }
    out->deltas[0] = L.x_delt.x; out->deltas[1] = L.x_delt.y; out->deltas[2] = L.x_delt.z;
    out->deltas[3] = L.y_delt.x; out->deltas[4] = L.y_delt.y; out->deltas[5] = L.y_delt.z;
    out->sub[0] = h_fdRectangleSubConstant.x;
    out->sub[1] = h_fdRectangleSubConstant.y;
    const FDLightPlaneParams &P = h_fdLightPlaneParams;
    out->lp_begin[0] = P.begin.x; out->lp_begin[1] = P.begin.y; out->lp_begin[2] = P.begin.z;
    out->lp_end[0] = P.end.x; out->lp_end[1] = P.end.y; out->lp_end[2] = P.end.z;
    out->lp_factor[0] = P.factor.x;
    out->lp_factor[1] = P.factor.y;
    std::memcpy(out->sample_aabb, sampleRectangleAABB, sizeof(out->sample_aabb));
    std::memcpy(out->model_aabb, modelRectangleAABB, sizeof(out->model_aabb));
    out->num_bins = FD_MAX_LP_GRID_SIZE * FD_MAX_LP_GRID_SIZE;
    out->valid_samples = m_validSampleNum;
    out->valid_tris = m_validTriangleNum;
    out->num_pairs = m_validBT_PairNum;
    out->view_log2up = log2up;
    out->errors = emu_error_count.load() + emu_surface_faults.load();

    const int NB = out->num_bins;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) out->shadow[(size_t)y * W + x] = pbo[((size_t)y << log2up) | x];
    auto cp = [](void *dst, const FD::Buffer<int> &b, size_t n) {
        if (dst && b.devPtr) std::memcpy(dst, b.devPtr, n);
    };
    if (out->sorted_keys) cp(out->sorted_keys, binSamplePairBinBuffer, 4ull * S);
    if (out->sorted_vals) cp(out->sorted_vals, binSamplePairSampleBuffer, 4ull * S);
    if (out->bin_sample_start) cp(out->bin_sample_start, binSampleStartBuffer, 4ull * (NB + 1));
    if (out->bin_sample_end) cp(out->bin_sample_end, binSampleEndBuffer, 4ull * (NB + 1));
    if (out->bin_maxz) std::memcpy(out->bin_maxz, binSampleMaxZBuffer.devPtr, 4ull * NB);
    if (out->bin_range) std::memcpy(out->bin_range, binSampleMinRangeBuffer.devPtr, 16ull * NB);
    if (out->tri_aabb) std::memcpy(out->tri_aabb, triAABBBuffer.devPtr, 32ull * in->T);
    if (out->tri_count) cp(out->tri_count, triPairNumBuffer, 4ull * in->T);
    if (out->tri_prefix) cp(out->tri_prefix, triPairNumPrefixSumBuffer, 4ull * in->T);
    const int np = m_validBT_PairNum < out->pair_capacity ? m_validBT_PairNum : out->pair_capacity;
    if (out->sorted_pair_bin && np > 0) cp(out->sorted_pair_bin, binTriPairBinBuffer, 4ull * np);
    if (out->sorted_pair_tri && np > 0) cp(out->sorted_pair_tri, binTriPairTriBuffer, 4ull * np);
    if (out->bin_tri_start) cp(out->bin_tri_start, binTriStartBuffer, 4ull * NB);
    if (out->bin_tri_end) cp(out->bin_tri_end, binTriEndBuffer, 4ull * NB);
    return 0;
}
