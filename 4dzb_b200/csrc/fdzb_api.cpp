// fdzb_api.cpp -- contexts, device arena and the extern "C" entry points.
//
// A context owns one scene (model 0), one view and one light, plus every
// scratch buffer of the pipeline, carved from a single grow-only device arena
// (the reference allocates the same buffers with FD::Buffer<T>,
// FS/api.cpp:48-144,205-294).  A frame is enqueued with no host round trip;
// fdzb_ctx_sync() reads back one small counter block, checks the device error
// word and, if the triangle/bin pair buffer overflowed, grows it and re-runs
// the frame (the reference has no such check, FS/constants.h:15).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/fdzb.h"
#include "fdzb_internal.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

#define FDZB_CUDA(call)                                                                        \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(FDZB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
    } while (0)

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

int ceil_log2(int v)
{
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}

struct Model {
    const float *vtx = nullptr;
    size_t nv = 0, strideBytes = 0;
    const int32_t *idx = nullptr;
    size_t nt = 0;
    std::string name;
};

}  // namespace

struct fdzb_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t ownStream = nullptr;
    // knobs (defaults of K/FourD.cu:61-62 and FS/constants.h:13)
    int cull = 1;
    float esp = 1e-6f;
    int bins = 16;
    int W = 0, H = 0;
    size_t maxTri = 0, maxVert = 0;
    const float4 *pos = nullptr, *nrm = nullptr;
    float *shadow = nullptr;
    uint32_t *masks = nullptr;
    std::vector<Model> models;
    bool lightSet = false;
    fdzb_area_light_desc lightDesc{};
    fdzb::LightParams light{};
    // device arena
    void *arena = nullptr;
    size_t arenaBytes = 0;
    fdzb::DeviceBuffers buf{};
    int pairCapacity = 0;
    uint32_t epoch = 0;
    int debug = 0;  // keep pre-sort copies for fdzb_ctx_export
    int triOrder = FDZB_TRI_ORDER_DEPTH;
    // pinned host staging
    fdzb::FrameDesc *hFrame = nullptr;
    fdzb::Counters *hCounters = nullptr;
    fdzb::FrameState *hState = nullptr;
    int *hBases = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool profile = false;  // record events at the stage boundaries
    cudaEvent_t stageEv[fdzb::STAGE_COUNT + 1] = {};
    int launches = 0;
    bool pending = false;
    fdzb_frame_stats stats{};
    float lastMs = 0.f;
};

namespace {

int ctx_check(fdzb_ctx *c)
{
    if (!c) return fail(FDZB_ERR_NOT_INITIALIZED, "context not initialised (call fdzb_init)");
    return FDZB_OK;
}

// Lays out every buffer of a launch of one frame inside the arena; returns bytes.
size_t layout(fdzb::DeviceBuffers &b, char *base, int S, int T, int NB, int P, bool debug)
{
    size_t off = 0;
    auto take = [&](size_t bytes) -> char * {
        off = align_up(off, 256);
        char *p = base ? base + off : nullptr;
        off += bytes;
        return p;
    };
    const int nf = 1;
    b.nframes = nf;
    b.totalSamples = S;
    b.totalTris = T;
    b.totalBins = NB;
    b.pairCapacity = P;
    b.frames = (fdzb::FrameDesc *)take(sizeof(fdzb::FrameDesc) * nf);
    b.states = (fdzb::FrameState *)take(sizeof(fdzb::FrameState) * nf);
    b.counters = (fdzb::Counters *)take(sizeof(fdzb::Counters));
    b.sortHist = (uint32_t *)take(sizeof(uint32_t) * 8 * 256);
    b.sampleBases = (int *)take(sizeof(int) * 3 * nf);
    b.triBases = b.sampleBases ? b.sampleBases + nf : nullptr;
    b.binBases = b.sampleBases ? b.sampleBases + 2 * nf : nullptr;
    const size_t Ss = (size_t)std::max(S, 1), Ts = (size_t)std::max(T, 1), Ps = (size_t)std::max(P, 1);
    b.keysA = (uint32_t *)take(4 * Ss);
    b.valsA = (uint32_t *)take(4 * Ss);
    b.keysB = (uint32_t *)take(4 * Ss);
    b.valsB = (uint32_t *)take(4 * Ss);
    b.binSampleStart = (int32_t *)take(4 * ((size_t)NB + 1));
    b.binSampleEnd = (int32_t *)take(4 * ((size_t)NB + 1));
    b.binStat = (uint32_t *)take(32 * (size_t)NB);
    b.triRec = (float4 *)take(64 * Ts);
    b.triCount = (int32_t *)take(4 * Ts);
    b.triScanStatus = (unsigned long long *)take(8 * ((Ts + fdzb::kTriTileHost - 1) / fdzb::kTriTileHost));
    b.pkeysA = (uint32_t *)take(4 * Ps);
    b.pvalsA = (uint32_t *)take(4 * Ps);
    b.pkeysB = (uint32_t *)take(4 * Ps);
    b.pvalsB = (uint32_t *)take(4 * Ps);
    b.binTriStart = (int32_t *)take(4 * (size_t)NB);
    b.binTriEnd = (int32_t *)take(4 * (size_t)NB);
    const size_t tiles = (std::max(Ss, Ps) + fdzb::kSortTileHost - 1) / fdzb::kSortTileHost;
    b.sortStatusTiles = tiles;
    b.sortStatus = (unsigned long long *)take(8 * 256 * tiles);
    b.itemCapacity = (int)(Ss / 32 + (size_t)NB + 1);
    b.items = (int4 *)take(16 * (size_t)b.itemCapacity);
    b.dbgKeys = b.dbgVals = b.dbgPKeys = b.dbgPVals = nullptr;
    if (debug) {
        b.dbgKeys = (uint32_t *)take(4 * Ss);
        b.dbgVals = (uint32_t *)take(4 * Ss);
        b.dbgPKeys = (uint32_t *)take(4 * Ps);
        b.dbgPVals = (uint32_t *)take(4 * Ps);
    }
    return align_up(off, 256);
}

int ensure_arena(fdzb_ctx *c, int S, int T, int NB, int P)
{
    fdzb::DeviceBuffers probe{};
    const size_t need = layout(probe, nullptr, S, T, NB, P, c->debug != 0);
    if (need > c->arenaBytes) {
        if (c->arena) {
            cudaStreamSynchronize(c->stream);
            cudaFree(c->arena);
            c->arena = nullptr;
            c->arenaBytes = 0;
        }
        const size_t bytes = align_up(need + need / 8, 1 << 20);
        cudaError_t e = cudaMalloc(&c->arena, bytes);
        if (e != cudaSuccess) {
            c->arena = nullptr;
            cudaGetLastError();
            return fail(FDZB_ERR_NO_MEMORY, "device arena of " + std::to_string(bytes) +
                                                " bytes: " + cudaGetErrorString(e));
        }
        c->arenaBytes = bytes;
        // look-back status words are epoch-tagged; start from a clean slate
        FDZB_CUDA(cudaMemsetAsync(c->arena, 0, bytes, c->stream));
    }
    layout(c->buf, (char *)c->arena, S, T, NB, P, c->debug != 0);
    return FDZB_OK;
}

int ready(fdzb_ctx *c)
{
    if (c->W <= 0 || c->H <= 0) return fail(FDZB_ERR_NOT_READY, "view size not set (fdzb_set_view)");
    if (!c->pos || !c->nrm) return fail(FDZB_ERR_NOT_READY, "sample buffers not set");
    if (!c->shadow) return fail(FDZB_ERR_NOT_READY, "output buffer not set");
    if (c->models.empty()) return fail(FDZB_ERR_NOT_READY, "no model added");
    if (!c->lightSet) return fail(FDZB_ERR_NOT_READY, "area light not set");
    return FDZB_OK;
}

int enqueue(fdzb_ctx *c)
{
    int rc = ready(c);
    if (rc) return rc;
    const Model &m = c->models[0];
    const long long S = (long long)c->W * c->H;
    if (S > 0x7fffffffll / 2) return fail(FDZB_ERR_INVALID_ARG, "view too large");
    if (m.nt > 0x3fffffffull || m.nv > 0x3fffffffull) return fail(FDZB_ERR_INVALID_ARG, "model too large");
    const int T = (int)m.nt, V = (int)m.nv;
    const int NB = c->bins * c->bins;
    if (c->pairCapacity <= 0) {
        long long guess = std::max<long long>(1 << 20, (long long)T * 64);
        c->pairCapacity = (int)std::min<long long>(guess, 1ll << 29);
    }
    rc = ensure_arena(c, (int)S, T, NB, c->pairCapacity);
    if (rc) return rc;
    fdzb::DeviceBuffers &b = c->buf;
    b.samplePasses = fdzb::sort_passes_for((long long)NB + 1);
    // Triangle lists: reference order sorts pairs by bin only (stable, so ascending
    // triangle id inside a bin, K/Step4_RasterizeTriangleToBin.inl:220-223).  Depth
    // order appends a depth bucket below the bin so each bin lists its lowest
    // triangles first, which fills the masks in far fewer pair tests; it uses the
    // key bits left over in the last radix pass, at least 4.
    {
        int binBits = 0;
        while ((1ll << binBits) < (long long)NB) ++binBits;
        if (c->triOrder == FDZB_TRI_ORDER_DEPTH) {
            const int passes = (binBits + 4 + 7) / 8;
            b.depthBits = std::min(10, passes * 8 - binBits);
        } else {
            b.depthBits = 0;
        }
        b.pairPasses = fdzb::sort_passes_for((long long)NB << b.depthBits);
    }
    b.epoch = ++c->epoch;

    fdzb::FrameDesc &f = *c->hFrame;
    std::memset(&f, 0, sizeof(f));
    f.pos = c->pos;
    f.nrm = c->nrm;
    f.vtx = m.vtx;
    f.idx = m.idx;
    f.shadow = c->shadow;
    f.masks = c->masks;
    f.W = c->W;
    f.H = c->H;
    f.log2up = ceil_log2(c->W);
    f.V = V;
    f.vstride = (int)(m.strideBytes / 4);
    f.T = T;
    f.Wb = c->bins;
    f.log2Wb = ceil_log2(c->bins);
    f.numBins = NB;
    f.cull = c->cull;
    f.esp = c->esp;
    f.maskWords = (c->light.N * c->light.N + 31) / 32;
    f.sampleBase = 0;
    f.triBase = 0;
    f.binBase = 0;
    f.light = c->light;
    c->hBases[0] = 0;
    c->hBases[1] = 0;
    c->hBases[2] = 0;

    FDZB_CUDA(cudaMemcpyAsync(b.frames, c->hFrame, sizeof(fdzb::FrameDesc), cudaMemcpyHostToDevice, c->stream));
    FDZB_CUDA(cudaMemcpyAsync(b.sampleBases, c->hBases, 3 * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    FDZB_CUDA(cudaMemsetAsync(b.counters, 0, sizeof(fdzb::Counters), c->stream));
    FDZB_CUDA(cudaMemsetAsync(b.sortHist, 0, 8 * 256 * sizeof(uint32_t), c->stream));
    FDZB_CUDA(cudaEventRecord(c->ev0, c->stream));
    FDZB_CUDA(fdzb::run_pipeline(b, (int)S, T, V, c->stream, c->profile ? c->stageEv : nullptr,
                                 &c->launches));
    FDZB_CUDA(cudaEventRecord(c->ev1, c->stream));
    FDZB_CUDA(cudaMemcpyAsync(c->hCounters, b.counters, sizeof(fdzb::Counters), cudaMemcpyDeviceToHost, c->stream));
    FDZB_CUDA(cudaMemcpyAsync(c->hState, b.states, sizeof(fdzb::FrameState), cudaMemcpyDeviceToHost, c->stream));
    c->pending = true;
    return FDZB_OK;
}

int sync_frame(fdzb_ctx *c)
{
    if (!c->pending) return FDZB_OK;
    int replans = 0;
    for (;;) {
        FDZB_CUDA(cudaStreamSynchronize(c->stream));
        c->pending = false;
        const fdzb::Counters &k = *c->hCounters;
        if (k.errorFlags & fdzb::ERR_LOOKBACK_TIMEOUT)
            return fail(FDZB_ERR_DEVICE_TIMEOUT, "a look-back wait exceeded its spin limit");
        if (k.errorFlags & fdzb::ERR_MBAR_TIMEOUT)
            return fail(FDZB_ERR_DEVICE_TIMEOUT, "a shared-memory barrier wait exceeded its limit");
        if (k.errorFlags & fdzb::ERR_BAD_INPUT)
            return fail(FDZB_ERR_INVALID_ARG, "triangle index out of range of the vertex buffer");
        if (k.errorFlags & fdzb::ERR_INTERNAL)
            return fail(FDZB_ERR_CUDA, "internal consistency check failed on the device");
        if (!k.pairOverflow) break;
        if (replans >= 3 || k.pairCount >= (1 << 29))
            return fail(FDZB_ERR_CAPACITY, "triangle/bin pair buffer overflow (" +
                                               std::to_string(k.pairCount) + " pairs)");
        c->pairCapacity = (int)std::min<long long>((long long)k.pairCount + k.pairCount / 4 + 1024, 1ll << 29);
        ++replans;
        int rc = enqueue(c);
        if (rc) return rc;
    }
    float ms = 0.f;
    FDZB_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->lastMs = ms;
    const fdzb::FrameState &s = *c->hState;
    const fdzb::Counters &k = *c->hCounters;
    fdzb_frame_stats &o = c->stats;
    std::memset(&o, 0, sizeof(o));
    o.state = (s.state == 2 && s.nValidTris == 0) ? 1 : s.state;
    o.valid_samples = o.state == 2 ? s.nValidSamples : 0;
    o.valid_triangles = s.state == 2 ? s.nValidTris : 0;
    o.num_pairs = o.state == 2 ? k.pairCount : 0;
    o.num_bins = c->bins * c->bins;
    o.pair_capacity = c->pairCapacity;
    o.pair_tests = (int64_t)k.pairTests;
    o.f = s.f;
    o.sub[0] = s.subx;
    o.sub[1] = s.suby;
    o.lp_begin[0] = s.Bx; o.lp_begin[1] = s.By; o.lp_begin[2] = s.Bz;
    o.lp_end[0] = s.Ex; o.lp_end[1] = s.Ey; o.lp_end[2] = s.Ez;
    o.lp_factor[0] = s.fx; o.lp_factor[1] = s.fy;
    for (int i = 0; i < 6; ++i) {
        o.sample_aabb[i] = s.sampleAabb[i];
        o.model_aabb[i] = s.modelAabb[i];
    }
    o.replans = replans;
    o.quirk_key_range = s.quirkKeyRange;
    o.kernel_launches = c->launches;
    o.rows_evaluated = (int64_t)k.rowsEvaluated;
    o.partial_masks = (int64_t)k.partialMasks;
    for (int i = 0; i < fdzb::STAGE_COUNT; ++i) {
        float t = 0.f;
        if (c->profile) cudaEventElapsedTime(&t, c->stageEv[i], c->stageEv[i + 1]);
        o.stage_ms[i] = t;
    }
    return FDZB_OK;
}

int ctx_init_resources(fdzb_ctx *c, int device)
{
    if (device < 0) {
        FDZB_CUDA(cudaGetDevice(&c->device));
    } else {
        c->device = device;
    }
    FDZB_CUDA(cudaSetDevice(c->device));
    FDZB_CUDA(cudaStreamCreateWithFlags(&c->ownStream, cudaStreamNonBlocking));
    c->stream = c->ownStream;
    FDZB_CUDA(cudaEventCreate(&c->ev0));
    FDZB_CUDA(cudaEventCreate(&c->ev1));
    for (auto &e : c->stageEv) FDZB_CUDA(cudaEventCreate(&e));
    FDZB_CUDA(cudaMallocHost(&c->hFrame, sizeof(fdzb::FrameDesc)));
    FDZB_CUDA(cudaMallocHost(&c->hCounters, sizeof(fdzb::Counters)));
    FDZB_CUDA(cudaMallocHost(&c->hState, sizeof(fdzb::FrameState)));
    FDZB_CUDA(cudaMallocHost(&c->hBases, 4 * sizeof(int)));
    return FDZB_OK;
}

void ctx_release(fdzb_ctx *c)
{
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->arena) cudaFree(c->arena);
    if (c->hFrame) cudaFreeHost(c->hFrame);
    if (c->hCounters) cudaFreeHost(c->hCounters);
    if (c->hState) cudaFreeHost(c->hState);
    if (c->hBases) cudaFreeHost(c->hBases);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    for (auto &e : c->stageEv)
        if (e) cudaEventDestroy(e);
    if (c->ownStream) cudaStreamDestroy(c->ownStream);
    delete c;
}

fdzb_ctx *g_ctx = nullptr;

bool is_device_pointer(const void *p)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

int fdzb::set_error(int code, const std::string &msg) { return fail(code, msg); }

extern "C" {

const char *fdzb_last_error(void) { return g_err.c_str(); }
const char *fdzb_version(void) { return "fdzb-b200 0.1 (sm_100a)"; }

int fdzb_ctx_create(fdzb_ctx **out, int device)
{
    if (!out) return fail(FDZB_ERR_INVALID_ARG, "out is NULL");
    fdzb_ctx *c = new (std::nothrow) fdzb_ctx();
    if (!c) return fail(FDZB_ERR_NO_MEMORY, "host allocation failed");
    int rc = ctx_init_resources(c, device);
    if (rc) {
        ctx_release(c);
        return rc;
    }
    *out = c;
    return FDZB_OK;
}

int fdzb_ctx_destroy(fdzb_ctx *c)
{
    ctx_release(c);
    return FDZB_OK;
}

int fdzb_ctx_set_stream(fdzb_ctx *c, void *stream)
{
    if (int rc = ctx_check(c)) return rc;
    c->stream = stream ? (cudaStream_t)stream : c->ownStream;
    return FDZB_OK;
}

int fdzb_ctx_set_debug(fdzb_ctx *c, int flags)
{
    if (int rc = ctx_check(c)) return rc;
    c->debug = flags & 1;
    return FDZB_OK;
}

int fdzb_ctx_set_profiling(fdzb_ctx *c, int enable)
{
    if (int rc = ctx_check(c)) return rc;
    c->profile = enable != 0;
    return FDZB_OK;
}

int fdzb_measure_alu_rate(double *lane_ops_per_second)
{
    if (!lane_ops_per_second) return fail(FDZB_ERR_INVALID_ARG, "out is NULL");
    FDZB_CUDA(fdzb::measure_alu_rate(lane_ops_per_second));
    return FDZB_OK;
}

int fdzb_ctx_set_tri_order(fdzb_ctx *c, int order)
{
    if (int rc = ctx_check(c)) return rc;
    if (order != FDZB_TRI_ORDER_REFERENCE && order != FDZB_TRI_ORDER_DEPTH)
        return fail(FDZB_ERR_INVALID_ARG, "unknown triangle order");
    c->triOrder = order;
    return FDZB_OK;
}

int fdzb_ctx_set_backface_cull(fdzb_ctx *c, int enable)
{
    if (int rc = ctx_check(c)) return rc;
    c->cull = enable ? 1 : 0;
    return FDZB_OK;
}

int fdzb_ctx_add_model(fdzb_ctx *c, const float *d_vtx, size_t n_vtx, size_t stride, const int32_t *d_idx,
                       size_t n_tri, const char *name)
{
    if (int rc = ctx_check(c)) return rc;
    if ((n_vtx && !d_vtx) || (n_tri && !d_idx)) return fail(FDZB_ERR_INVALID_ARG, "NULL model buffer");
    if (stride < 12 || stride % 4) return fail(FDZB_ERR_INVALID_ARG, "vertex stride must be >= 12 and a multiple of 4 bytes");
    Model m;
    m.vtx = d_vtx;
    m.nv = n_vtx;
    m.strideBytes = stride;
    m.idx = d_idx;
    m.nt = n_tri;
    m.name = name ? name : "";
    c->models.push_back(m);
    return FDZB_OK;
}

int fdzb_ctx_set_sample_buffers(fdzb_ctx *c, const float *d_pos, const float *d_nrm)
{
    if (int rc = ctx_check(c)) return rc;
    if (((uintptr_t)d_pos & 15) || ((uintptr_t)d_nrm & 15))
        return fail(FDZB_ERR_INVALID_ARG, "sample buffers must be 16-byte aligned float4 arrays");
    c->pos = (const float4 *)d_pos;
    c->nrm = (const float4 *)d_nrm;
    return FDZB_OK;
}

int fdzb_ctx_set_output_buffer(fdzb_ctx *c, float *d_shadow, uint32_t *d_masks)
{
    if (int rc = ctx_check(c)) return rc;
    c->shadow = d_shadow;
    c->masks = d_masks;
    return FDZB_OK;
}

int fdzb_ctx_set_bin_num(fdzb_ctx *c, size_t n)
{
    if (int rc = ctx_check(c)) return rc;
    if (n < 1 || n > (size_t)fdzb::kMaxBins || (n & (n - 1)))
        return fail(FDZB_ERR_INVALID_ARG, "bin number must be a power of two in [1, 512]");
    c->bins = (int)n;
    return FDZB_OK;
}

int fdzb_ctx_set_view(fdzb_ctx *c, int w, int h)
{
    if (int rc = ctx_check(c)) return rc;
    if (w <= 0 || h <= 0 || (long long)w * h > (1ll << 30)) return fail(FDZB_ERR_INVALID_ARG, "bad view size");
    c->W = w;
    c->H = h;
    return FDZB_OK;
}

int fdzb_ctx_set_scenes_esp(fdzb_ctx *c, float esp)
{
    if (int rc = ctx_check(c)) return rc;
    c->esp = esp;
    return FDZB_OK;
}

int fdzb_ctx_set_scene_params(fdzb_ctx *c, size_t maxTri, size_t maxVert)
{
    if (int rc = ctx_check(c)) return rc;
    c->maxTri = maxTri;
    c->maxVert = maxVert;
    return FDZB_OK;
}

int fdzb_ctx_set_area_light(fdzb_ctx *c, const fdzb_area_light_desc *d)
{
    if (int rc = ctx_check(c)) return rc;
    if (!d) return fail(FDZB_ERR_INVALID_ARG, "light is NULL");
    if (d->lightResWidth != d->lightResHeight || d->lightResWidth < 1 || d->lightResWidth > fdzb::kMaxLightN)
        return fail(FDZB_ERR_UNSUPPORTED, "light grid must be square with N in [1, 32]");
    c->lightDesc = *d;
    fdzb::light_setup(d->rightRadius, d->topRadius, d->position, d->viewDir, d->upDir, d->lightResWidth,
                      d->lightResHeight, &c->light);
    c->lightSet = true;
    return FDZB_OK;
}

int fdzb_ctx_move_model(fdzb_ctx *c, const float m[16])
{
    if (int rc = ctx_check(c)) return rc;
    if (!m) return fail(FDZB_ERR_INVALID_ARG, "matrix is NULL");
    if (c->models.empty()) return fail(FDZB_ERR_NOT_READY, "no model added");
    if (int rc = sync_frame(c)) return rc;
    const Model &md = c->models[0];
    FDZB_CUDA(fdzb::run_move_model(const_cast<float *>(md.vtx), (int)(md.strideBytes / 4), (int)md.nv, m, c->stream));
    FDZB_CUDA(cudaStreamSynchronize(c->stream));
    return FDZB_OK;
}

int fdzb_ctx_launch_async(fdzb_ctx *c)
{
    if (int rc = ctx_check(c)) return rc;
    if (c->pending) {
        int rc = sync_frame(c);
        if (rc) return rc;
    }
    return enqueue(c);
}

int fdzb_ctx_sync(fdzb_ctx *c)
{
    if (int rc = ctx_check(c)) return rc;
    return sync_frame(c);
}

int fdzb_ctx_launch(fdzb_ctx *c, float *ms)
{
    int rc = fdzb_ctx_launch_async(c);
    if (rc) return rc;
    rc = sync_frame(c);
    if (rc) return rc;
    if (ms) *ms = c->lastMs;
    return FDZB_OK;
}

int fdzb_ctx_get_stats(fdzb_ctx *c, fdzb_frame_stats *out)
{
    if (int rc = ctx_check(c)) return rc;
    if (!out) return fail(FDZB_ERR_INVALID_ARG, "out is NULL");
    *out = c->stats;
    return FDZB_OK;
}

int fdzb_ctx_export(fdzb_ctx *c, int what, void *dst, size_t bytes)
{
    if (int rc = ctx_check(c)) return rc;
    if (!dst) return fail(FDZB_ERR_INVALID_ARG, "dst is NULL");
    if (!c->arena) return fail(FDZB_ERR_NOT_READY, "no launch yet");
    if (int rc = sync_frame(c)) return rc;
    const fdzb::DeviceBuffers &b = c->buf;
    const size_t S = (size_t)b.totalSamples, T = (size_t)b.totalTris, NB = (size_t)b.totalBins;
    const size_t P = (size_t)std::min(c->hCounters->pairCount, b.pairCapacity);
    const bool sOdd = b.samplePasses & 1, pOdd = b.pairPasses & 1;
    const void *src = nullptr;
    size_t avail = 0;
    std::vector<char> tmp;
    switch (what) {
    case FDZB_ARR_SAMPLE_KEYS:
        if (!b.dbgKeys) return fail(FDZB_ERR_NOT_READY, "pre-sort arrays need fdzb_ctx_set_debug(ctx, 1)");
        src = b.dbgKeys; avail = 4 * S; break;
    case FDZB_ARR_SORTED_SAMPLE_KEYS: src = sOdd ? b.keysB : b.keysA; avail = 4 * S; break;
    case FDZB_ARR_SORTED_SAMPLE_IDS: src = sOdd ? b.valsB : b.valsA; avail = 4 * S; break;
    case FDZB_ARR_BIN_SAMPLE_START: src = b.binSampleStart; avail = 4 * (NB + 1); break;
    case FDZB_ARR_BIN_SAMPLE_END: src = b.binSampleEnd; avail = 4 * (NB + 1); break;
    case FDZB_ARR_BIN_MAXZ:
    case FDZB_ARR_BIN_RANGE: {
        std::vector<uint32_t> raw(8 * NB);
        FDZB_CUDA(cudaMemcpy(raw.data(), b.binStat, 32 * NB, cudaMemcpyDeviceToHost));
        auto dec = [](uint32_t o) {
            uint32_t u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
            float f;
            std::memcpy(&f, &u, 4);
            return f;
        };
        const size_t n = what == FDZB_ARR_BIN_MAXZ ? NB : 4 * NB;
        tmp.resize(4 * n);
        float *o = (float *)tmp.data();
        for (size_t i = 0; i < NB; ++i) {
            if (what == FDZB_ARR_BIN_MAXZ) o[i] = dec(raw[8 * i]);
            else for (int k = 0; k < 4; ++k) o[4 * i + k] = dec(raw[8 * i + 1 + k]);
        }
        if (bytes > tmp.size()) return fail(FDZB_ERR_INVALID_ARG, "export size exceeds the array");
        std::memcpy(dst, tmp.data(), bytes);
        return FDZB_OK;
    }
    case FDZB_ARR_TRI_COUNT: src = b.triCount; avail = 4 * T; break;
    case FDZB_ARR_PAIR_BIN:
    case FDZB_ARR_SORTED_PAIR_BIN: {
        // pair keys carry the depth bucket below the bin; export the bin
        const uint32_t *s2 = what == FDZB_ARR_PAIR_BIN ? b.dbgPKeys : (pOdd ? b.pkeysB : b.pkeysA);
        if (!s2) return fail(FDZB_ERR_NOT_READY, "pre-sort arrays need fdzb_ctx_set_debug(ctx, 1)");
        if (bytes > 4 * P) return fail(FDZB_ERR_INVALID_ARG, "export size exceeds the array");
        std::vector<uint32_t> v(bytes / 4);
        if (!v.empty()) FDZB_CUDA(cudaMemcpy(v.data(), s2, 4 * v.size(), cudaMemcpyDeviceToHost));
        for (uint32_t &x : v) x >>= b.depthBits;
        std::memcpy(dst, v.data(), 4 * v.size());
        return FDZB_OK;
    }
    case FDZB_ARR_PAIR_TRI:
        if (!b.dbgPVals) return fail(FDZB_ERR_NOT_READY, "pre-sort arrays need fdzb_ctx_set_debug(ctx, 1)");
        src = b.dbgPVals; avail = 4 * P; break;
    case FDZB_ARR_SORTED_PAIR_TRI: src = pOdd ? b.pvalsB : b.pvalsA; avail = 4 * P; break;
    case FDZB_ARR_BIN_TRI_START: src = b.binTriStart; avail = 4 * NB; break;
    case FDZB_ARR_BIN_TRI_END: src = b.binTriEnd; avail = 4 * NB; break;
    case FDZB_ARR_TRI_AABB: {
        std::vector<float4> rec(4 * T);
        if (T) FDZB_CUDA(cudaMemcpy(rec.data(), b.triRec, 64 * T, cudaMemcpyDeviceToHost));
        tmp.resize(32 * T);
        float *o = (float *)tmp.data();
        for (size_t t = 0; t < T; ++t) {
            const float4 q0 = rec[4 * t], q1 = rec[4 * t + 1], q3 = rec[4 * t + 3];
            const float v[8] = {q3.x, q3.y, q0.w, 1.0f, q3.z, q3.w, q1.w, 1.0f};
            std::memcpy(o + 8 * t, v, 32);
        }
        if (bytes > tmp.size()) return fail(FDZB_ERR_INVALID_ARG, "export size exceeds the array");
        std::memcpy(dst, tmp.data(), bytes);
        return FDZB_OK;
    }
    default: return fail(FDZB_ERR_INVALID_ARG, "unknown array id");
    }
    if (bytes > avail) return fail(FDZB_ERR_INVALID_ARG, "export size exceeds the array");
    if (bytes) FDZB_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return FDZB_OK;
}

int fdzb_light_setup(const fdzb_area_light_desc *d, float mat[16], float rf[2], float corners[12], float deltas[6])
{
    if (!d) return fail(FDZB_ERR_INVALID_ARG, "light is NULL");
    if (d->lightResWidth < 1 || d->lightResHeight < 1) return fail(FDZB_ERR_INVALID_ARG, "bad light grid");
    fdzb::LightParams L;
    fdzb::light_setup(d->rightRadius, d->topRadius, d->position, d->viewDir, d->upDir, d->lightResWidth,
                      d->lightResHeight, &L);
    if (mat) std::memcpy(mat, L.mat, sizeof(L.mat));
    if (rf) std::memcpy(rf, L.RF, sizeof(L.RF));
    if (corners) {
        std::memcpy(corners, L.ur, 12);
        std::memcpy(corners + 3, L.ul, 12);
        std::memcpy(corners + 6, L.dl, 12);
        std::memcpy(corners + 9, L.dr, 12);
    }
    if (deltas) {
        std::memcpy(deltas, L.xd, 12);
        std::memcpy(deltas + 3, L.yd, 12);
    }
    return FDZB_OK;
}

// ---- reference-shaped global context -----------------------------------------

int fdzb_init(void)
{
    if (g_ctx) {
        ctx_release(g_ctx);
        g_ctx = nullptr;
    }
    return fdzb_ctx_create(&g_ctx, -1);
}
int fdzb_set_backface_cull(int enable) { return fdzb_ctx_set_backface_cull(g_ctx, enable); }
int fdzb_add_model(const float *d_vtx, size_t n_vtx, size_t stride, const int32_t *d_idx, size_t n_tri,
                   const char *name)
{
    return fdzb_ctx_add_model(g_ctx, d_vtx, n_vtx, stride, d_idx, n_tri, name);
}
int fdzb_set_sample_buffers(const float *d_pos, const float *d_nrm)
{
    return fdzb_ctx_set_sample_buffers(g_ctx, d_pos, d_nrm);
}
int fdzb_set_output_buffer(float *d_shadow, uint32_t *d_masks)
{
    return fdzb_ctx_set_output_buffer(g_ctx, d_shadow, d_masks);
}
int fdzb_register_resources(void)
{
    if (int rc = ctx_check(g_ctx)) return rc;
    fdzb_ctx *c = g_ctx;
    if (c->pos && !is_device_pointer(c->pos)) return fail(FDZB_ERR_INVALID_ARG, "sample position buffer is not device memory");
    if (c->nrm && !is_device_pointer(c->nrm)) return fail(FDZB_ERR_INVALID_ARG, "sample normal buffer is not device memory");
    if (c->shadow && !is_device_pointer(c->shadow)) return fail(FDZB_ERR_INVALID_ARG, "output buffer is not device memory");
    for (const Model &m : c->models)
        if ((m.vtx && !is_device_pointer(m.vtx)) || (m.idx && !is_device_pointer(m.idx)))
            return fail(FDZB_ERR_INVALID_ARG, "model buffer is not device memory");
    return FDZB_OK;
}
int fdzb_unregister_resources(void) { return ctx_check(g_ctx); }
int fdzb_set_bin_num(size_t n) { return fdzb_ctx_set_bin_num(g_ctx, n); }
int fdzb_set_view(int w, int h) { return fdzb_ctx_set_view(g_ctx, w, h); }
int fdzb_set_scenes_esp(float esp) { return fdzb_ctx_set_scenes_esp(g_ctx, esp); }
int fdzb_set_scene_params(size_t maxTri, size_t maxVert) { return fdzb_ctx_set_scene_params(g_ctx, maxTri, maxVert); }
int fdzb_set_area_light(const fdzb_area_light_desc *d) { return fdzb_ctx_set_area_light(g_ctx, d); }
float fdzb_launch(void)
{
    float ms = 0.f;
    int rc = fdzb_ctx_launch(g_ctx, &ms);
    return rc ? (float)rc : ms;
}
int fdzb_move_model(const float m[16]) { return fdzb_ctx_move_model(g_ctx, m); }

}  // extern "C"
