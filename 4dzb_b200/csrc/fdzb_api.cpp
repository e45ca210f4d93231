// fdzb_api.cpp -- engine, contexts, batches and the extern "C" entry points.
//
// An Engine owns every scratch buffer of the pipeline, carved from a single
// grow-only device arena (the reference allocates the same buffers with
// FD::Buffer<T>, FS/api.cpp:48-144,205-294), plus the pinned staging blocks and
// the CUDA graph of its last launch shape.  A launch processes a list of
// frames laid end to end in HBM (one frame for the FD-shaped context API, up to
// thousands for a batch) with no host round trip; sync reads back one small
// counter block, checks the device error word and, if the triangle/bin pair
// buffer overflowed, grows it and re-runs the launch (the reference has no such
// check, FS/constants.h:15).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/fdzb.h"
#include "fdzb_engine.h"
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

int ceil_log2(long long v)
{
    int l = 0;
    while ((1ll << l) < v) ++l;
    return l;
}

// ABI layouts mirrored by the ctypes binding
static_assert(sizeof(fdzb_area_light_desc) == 52, "fdzb_area_light_desc layout");
static_assert(sizeof(fdzb_frame_stats) == 184, "fdzb_frame_stats layout");
static_assert(sizeof(fdzb_frame_desc) == 152, "fdzb_frame_desc layout");
static_assert(sizeof(fdzb_batch_stats) == 232, "fdzb_batch_stats layout");
static_assert(sizeof(fdzb_shade_desc) == 120, "fdzb_shade_desc layout");

constexpr long long kMaxPairCapacity = 1ll << 29;
constexpr long long kMaxTotalSamples = 0x7fffffffll / 2;
constexpr long long kMaxTotalBins = 1ll << 27;
// coverage bucket of the triangle order: log2 of the angular size in steps of
// 1/25.6 octave (fdzb_pipeline.cu: coverage_bucket)
constexpr int kCoverageBucketBits = 10;

struct Model {
    const float *vtx = nullptr;
    size_t nv = 0, strideBytes = 0;
    const int32_t *idx = nullptr;
    size_t nt = 0;
    std::string name;
};

}  // namespace

namespace fdzb {

namespace {

// Lays out every buffer of a launch of nf frames inside the arena; returns bytes.
size_t layout(fdzb::DeviceBuffers &b, char *base, int nf, long long S, long long T, long long NB, long long P,
              bool debug)
{
    size_t off = 0;
    auto take = [&](size_t bytes) -> char * {
        off = align_up(off, 256);
        char *p = base ? base + off : nullptr;
        off += bytes;
        return p;
    };
    b.nframes = nf;
    b.totalSamples = (int)S;
    b.totalTris = (int)T;
    b.totalBins = (int)NB;
    b.pairCapacity = (int)P;
    b.frames = (fdzb::FrameDesc *)take(sizeof(fdzb::FrameDesc) * nf);
    b.states = (fdzb::FrameState *)take(sizeof(fdzb::FrameState) * nf);
    b.counters = (fdzb::Counters *)take(sizeof(fdzb::Counters));
    b.epochWord = (uint32_t *)take(sizeof(uint32_t));
    b.sortHist = (uint32_t *)take(sizeof(uint32_t) * 4 * fdzb::kSortSlots * 256);
    b.sampleBases = (int *)take(sizeof(int) * 3 * nf);
    b.triBases = b.sampleBases ? b.sampleBases + nf : nullptr;
    b.binBases = b.sampleBases ? b.sampleBases + 2 * nf : nullptr;
    const size_t Ss = (size_t)std::max(S, 1ll), Ts = (size_t)std::max(T, 1ll), Ps = (size_t)std::max(P, 1ll);
    b.keysA = (uint32_t *)take(4 * Ss);
    b.valsA = (uint32_t *)take(4 * Ss);
    b.keysB = (uint32_t *)take(4 * Ss);
    b.valsB = (uint32_t *)take(4 * Ss);
    b.binSampleStart = (int32_t *)take(4 * ((size_t)NB + 1));
    b.binSampleEnd = (int32_t *)take(4 * ((size_t)NB + 1));
    b.binStat = (uint32_t *)take(32 * (size_t)NB);
    b.triRec = (float4 *)take(64 * Ts);
    b.triPrj = (float4 *)take(32 * Ts);
    b.triCount = (int32_t *)take(4 * Ts);
    b.triScanStatus = (unsigned long long *)take(8 * ((Ts + fdzb::kTriTileHost - 1) / fdzb::kTriTileHost));
    b.tkeysA = (uint32_t *)take(4 * Ts);
    b.tvalsA = (uint32_t *)take(4 * Ts);
    b.tkeysB = (uint32_t *)take(4 * Ts);
    b.tvalsB = (uint32_t *)take(4 * Ts);
    b.pkeysA = (uint32_t *)take(4 * Ps);
    b.pvalsA = (uint32_t *)take(4 * Ps);
    b.pkeysB = (uint32_t *)take(4 * Ps);
    b.pvalsB = (uint32_t *)take(4 * Ps);
    b.binTriStart = (int32_t *)take(4 * (size_t)NB);
    b.binTriEnd = (int32_t *)take(4 * (size_t)NB);
    const size_t tiles = (std::max(std::max(Ss, Ps), Ts) + fdzb::kSortTileHost - 1) / fdzb::kSortTileHost;
    b.sortStatusTiles = tiles;
    b.sortStatus = (unsigned long long *)take(8 * 256 * tiles);
    b.itemCapacity = (int)(Ss / 32 + (size_t)NB + (size_t)nf + 1);
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

}  // namespace

void drop_graph(Engine &e)
{
    if (e.graph) cudaGraphExecDestroy(e.graph);
    e.graph = nullptr;
    e.graphKey = GraphKey{};
}

namespace {

int ensure_arena(Engine &e, int nf, long long S, long long T, long long NB, long long P)
{
    fdzb::DeviceBuffers probe{};
    const size_t need = layout(probe, nullptr, nf, S, T, NB, P, e.debug != 0);
    if (need > e.arenaBytes) {
        if (e.arena) {
            cudaStreamSynchronize(e.stream);
            drop_graph(e);
            cudaFree(e.arena);
            e.arena = nullptr;
            e.arenaBytes = 0;
        }
        const size_t bytes = align_up(need + need / 8, 1 << 20);
        cudaError_t err = cudaMalloc(&e.arena, bytes);
        if (err != cudaSuccess) {
            e.arena = nullptr;
            cudaGetLastError();
            return fail(FDZB_ERR_NO_MEMORY, "device arena of " + std::to_string(bytes) +
                                                " bytes: " + cudaGetErrorString(err));
        }
        e.arenaBytes = bytes;
        // look-back status words are tagged with the launch number; start clean
        FDZB_CUDA(cudaMemsetAsync(e.arena, 0, bytes, e.stream));
    }
    layout(e.buf, (char *)e.arena, nf, S, T, NB, P, e.debug != 0);
    return FDZB_OK;
}

int ensure_host(Engine &e, int nf)
{
    if (nf <= e.hCap) return FDZB_OK;
    if (e.pending) cudaStreamSynchronize(e.stream);
    drop_graph(e);
    if (e.hFrames) cudaFreeHost(e.hFrames);
    if (e.hStates) cudaFreeHost(e.hStates);
    if (e.hBases) cudaFreeHost(e.hBases);
    e.hFrames = nullptr;
    e.hStates = nullptr;
    e.hBases = nullptr;
    e.hCap = 0;
    const int cap = std::max(nf, 1);
    FDZB_CUDA(cudaMallocHost(&e.hFrames, sizeof(fdzb::FrameDesc) * cap));
    FDZB_CUDA(cudaMallocHost(&e.hStates, sizeof(fdzb::FrameState) * cap));
    FDZB_CUDA(cudaMallocHost(&e.hBases, sizeof(int) * 3 * cap));
    e.hCap = cap;
    return FDZB_OK;
}

}  // namespace

void engine_free_arena(Engine &e)
{
    if (e.stream) cudaStreamSynchronize(e.stream);
    e.pending = false;
    drop_graph(e);
    if (e.arena) cudaFree(e.arena);
    e.arena = nullptr;
    e.arenaBytes = 0;
}

int engine_init(Engine &e, int device)
{
    if (device < 0) {
        FDZB_CUDA(cudaGetDevice(&e.device));
    } else {
        e.device = device;
    }
    FDZB_CUDA(cudaSetDevice(e.device));
    FDZB_CUDA(cudaStreamCreateWithFlags(&e.ownStream, cudaStreamNonBlocking));
    e.stream = e.ownStream;
    FDZB_CUDA(cudaEventCreate(&e.ev0));
    FDZB_CUDA(cudaEventCreate(&e.ev1));
    for (auto &ev : e.stageEv) FDZB_CUDA(cudaEventCreate(&ev));
    FDZB_CUDA(cudaMallocHost(&e.hCounters, sizeof(fdzb::Counters)));
    return ensure_host(e, 1);
}

void engine_release(Engine &e)
{
    if (e.stream) cudaStreamSynchronize(e.stream);
    drop_graph(e);
    if (e.arena) cudaFree(e.arena);
    if (e.hFrames) cudaFreeHost(e.hFrames);
    if (e.hStates) cudaFreeHost(e.hStates);
    if (e.hBases) cudaFreeHost(e.hBases);
    if (e.hCounters) cudaFreeHost(e.hCounters);
    if (e.passMasks) cudaFree(e.passMasks);
    if (e.ev0) cudaEventDestroy(e.ev0);
    if (e.ev1) cudaEventDestroy(e.ev1);
    for (auto &ev : e.stageEv)
        if (ev) cudaEventDestroy(ev);
    if (e.ownStream) cudaStreamDestroy(e.ownStream);
    e = Engine{};
}

namespace {

// Checks one frame's inputs (the conditions FD:: assumes of its callers).
int check_frame(const FrameSpec &f, int i)
{
    const std::string at = "frame " + std::to_string(i) + ": ";
    if (f.W <= 0 || f.H <= 0 || (long long)f.W * f.H > (1ll << 30)) return fail(FDZB_ERR_INVALID_ARG, at + "bad view size");
    if (!f.pos || !f.nrm) return fail(FDZB_ERR_NOT_READY, at + "sample buffers not set");
    if (((uintptr_t)f.pos & 15) || ((uintptr_t)f.nrm & 15))
        return fail(FDZB_ERR_INVALID_ARG, at + "sample buffers must be 16-byte aligned float4 arrays");
    if (!f.shadow) return fail(FDZB_ERR_NOT_READY, at + "output buffer not set");
    if ((f.nv && !f.vtx) || (f.nt && !f.idx)) return fail(FDZB_ERR_INVALID_ARG, at + "NULL model buffer");
    if (f.strideBytes < 12 || f.strideBytes % 4)
        return fail(FDZB_ERR_INVALID_ARG, at + "vertex stride must be >= 12 and a multiple of 4 bytes");
    if (f.nt > 0x3fffffffull || f.nv > 0x3fffffffull) return fail(FDZB_ERR_INVALID_ARG, at + "model too large");
    if (f.bins < 1 || f.bins > fdzb::kMaxBins || (f.bins & (f.bins - 1)))
        return fail(FDZB_ERR_INVALID_ARG, at + "bin number must be a power of two in [1, 512]");
    if (f.light.N < 1 || f.light.N > fdzb::kMaxLightN || f.light.NC < 1 || f.light.NC > fdzb::kMaxLightN)
        return fail(FDZB_ERR_UNSUPPORTED, at + "light grid width and height must be in [1, 64]");
    if (!valid_occ_shape(f.occChunk, f.occItem))
        return fail(FDZB_ERR_INVALID_ARG, at + "occlusion shape: chunk in {8, 16, 32}, item in {32, 64, 128}");
    return FDZB_OK;
}

// Fills the pinned frame table and enqueues copies, the pipeline and the
// read-back of counters and frame states (captured into a graph or not).
cudaError_t enqueue_body(Engine &e, int nf)
{
    fdzb::DeviceBuffers &b = e.buf;
    cudaStream_t s = e.stream;
    cudaError_t err;
    if ((err = cudaMemcpyAsync(b.frames, e.hFrames, sizeof(fdzb::FrameDesc) * nf, cudaMemcpyHostToDevice, s))) return err;
    if ((err = cudaMemcpyAsync(b.sampleBases, e.hBases, 3 * sizeof(int) * nf, cudaMemcpyHostToDevice, s))) return err;
    if ((err = cudaMemsetAsync(b.counters, 0, sizeof(fdzb::Counters), s))) return err;
    if ((err = cudaMemsetAsync(b.sortHist, 0, 4 * fdzb::kSortSlots * 256 * sizeof(uint32_t), s))) return err;
    if ((err = fdzb::run_pipeline(b, e.maxS, e.maxT, e.maxV, s, e.profile ? e.stageEv : nullptr, &e.launches))) return err;
    if ((err = cudaMemcpyAsync(e.hCounters, b.counters, sizeof(fdzb::Counters), cudaMemcpyDeviceToHost, s))) return err;
    return cudaMemcpyAsync(e.hStates, b.states, sizeof(fdzb::FrameState) * nf, cudaMemcpyDeviceToHost, s);
}

// Clears the look-back status words and the epoch word when the arena's layout
// moved them or the launch count reached kEpochLimit, then counts this launch.
// Enqueued on the engine's stream before the launch, outside any graph.
cudaError_t refresh_lookback(Engine &e)
{
    const fdzb::DeviceBuffers &b = e.buf;
    const auto where = std::make_tuple((const void *)b.sortStatus, b.sortStatusTiles, (const void *)b.triScanStatus,
                                       b.totalTris, (const void *)b.epochWord);
    if (where != e.statusLayout || e.epochCount >= kEpochLimit) {
        const size_t triTiles = ((size_t)std::max(b.totalTris, 1) + fdzb::kTriTileHost - 1) / fdzb::kTriTileHost;
        cudaError_t err;
        if ((err = cudaMemsetAsync(b.sortStatus, 0, 8 * 256 * b.sortStatusTiles, e.stream))) return err;
        if ((err = cudaMemsetAsync(b.triScanStatus, 0, 8 * triTiles, e.stream))) return err;
        if ((err = cudaMemsetAsync(b.epochWord, 0, sizeof(uint32_t), e.stream))) return err;
        e.epochCount = 0;
        e.statusLayout = where;
    }
    ++e.epochCount;
    return cudaSuccess;
}

}  // namespace

int engine_enqueue(Engine &e)
{
    const int nf = (int)e.frames.size();
    if (nf <= 0) return fail(FDZB_ERR_INVALID_ARG, "no frames");
    long long S = 0, T = 0, NB = 0;
    int maxS = 0, maxT = 0, maxV = 0;
    for (int i = 0; i < nf; ++i) {
        const FrameSpec &f = e.frames[i];
        if (int rc = check_frame(f, i)) return rc;
        const long long s = (long long)f.W * f.H;
        S += s;
        T += (long long)f.nt;
        NB += (long long)f.bins * f.bins;
        maxS = std::max<int>(maxS, (int)s);
        maxT = std::max<int>(maxT, (int)f.nt);
        maxV = std::max<int>(maxV, (int)f.nv);
    }
    if (S > kMaxTotalSamples) return fail(FDZB_ERR_INVALID_ARG, "too many samples in one launch");
    if (T > 0x3fffffffll) return fail(FDZB_ERR_INVALID_ARG, "too many triangles in one launch");
    if (NB > kMaxTotalBins) return fail(FDZB_ERR_INVALID_ARG, "too many light-plane bins in one launch");
    if (nf > 65535) return fail(FDZB_ERR_INVALID_ARG, "too many frames in one launch (max 65535)");
    if (e.pairCapacity <= 0) e.pairCapacity = std::min(default_pair_capacity(T), e.maxPairCapacity);
    if (int rc = ensure_host(e, nf)) return rc;
    if (int rc = ensure_arena(e, nf, S, T, NB, e.pairCapacity)) return rc;
    e.maxS = maxS;
    e.maxT = maxT;
    e.maxV = maxV;
    fdzb::DeviceBuffers &b = e.buf;
    b.samplePasses = fdzb::sort_passes_for(NB + 1);
    // 64-bit row words when some frame's grid exceeds 32 rows or columns; the
    // lane-per-pair schedule covers square 32-bit grids without the depth
    // plane, other launches use lane per sample
    bool wide = false, square = true, rows16 = true;
    for (const FrameSpec &f : e.frames) {
        wide = wide || f.light.N > fdzb::kMaxLightN32 || f.light.NC > fdzb::kMaxLightN32;
        square = square && f.light.N == f.light.NC;
        rows16 = rows16 && f.light.N <= 16;
    }
    b.wide = wide ? 1 : 0;
    b.rows16 = rows16 ? 1 : 0;
    b.depthPlane = e.depthPlane;
    b.rayCast = e.rayCast;
    b.occVariant = (e.occVariant == 1 && !wide && square && !e.depthPlane) ? 1 : 0;
    {
        e.lastShape = std::make_tuple(nf, S, T, NB);
        const auto known = e.openBoxKeep.find(e.lastShape);   // a shape not seen yet: probe the cull
        const bool want = e.openBoxMode == FDZB_OPEN_BOX_ON ||
                          (e.openBoxMode == FDZB_OPEN_BOX_AUTO && (known == e.openBoxKeep.end() || known->second));
        b.openBox = (want && !e.rayCast && b.occVariant == 0) ? 1 : 0;
        b.countWork = (e.profile && e.countWork) ? 1 : 0;
        e.lastOpenBox = b.openBox != 0;
    }
    // Triangle lists: the pairs are sorted by bin only (stable, so a bin lists
    // its triangles in the order the pairs were emitted,
    // K/Step4_RasterizeTriangleToBin.inl:220-223).  Reference order emits them by
    // ascending triangle id; coverage order first sorts the triangles (stably) by
    // a coverage bucket and emits them in that order, so each bin lists its
    // widest triangles first, which fills the masks in far fewer pair tests.
    b.depthBits = e.triOrder == FDZB_TRI_ORDER_COVERAGE ? kCoverageBucketBits : 0;
    b.triPasses = b.depthBits ? fdzb::sort_passes_for(1ll << b.depthBits) : 0;
    b.pairPasses = fdzb::sort_passes_for(NB);
    // A pair is one word, bin << triBits | triangle, when the bin and triangle
    // numbers fit 32 bits together (the HD frame: 14 + 18): the pair sort then
    // moves keys alone, half the bytes and instructions of a key/value sort,
    // on the same digits (bits triBits and up), and keeps the same order.
    {
        auto bitsFor = [](long long n) {
            int k = 1;
            while (k < 32 && (1ll << k) < n) ++k;
            return k;
        };
        const int binBits = bitsFor((long long)NB), triBits = bitsFor((long long)T);
        b.pairTriBits = (!e.separatePairs && binBits + triBits <= 32) ? triBits : 0;
    }
    int sb = 0, tb = 0, bb = 0;
    for (int i = 0; i < nf; ++i) {
        const FrameSpec &s = e.frames[i];
        fdzb::FrameDesc &f = e.hFrames[i];
        std::memset(&f, 0, sizeof(f));
        f.pos = s.pos;
        f.nrm = s.nrm;
        f.vtx = s.vtx;
        f.idx = s.idx;
        f.shadow = s.shadow;
        f.masks = s.masks;
        f.W = s.W;
        f.H = s.H;
        f.log2up = ceil_log2(s.W);
        f.V = (int)s.nv;
        f.vstride = (int)(s.strideBytes / 4);
        f.T = (int)s.nt;
        f.Wb = s.bins;
        f.log2Wb = ceil_log2(s.bins);
        f.numBins = s.bins * s.bins;
        f.cull = s.cull;
        f.esp = s.esp;
        f.maskWords = (s.light.N * s.light.NC + 31) / 32;
        f.sampleBase = sb;
        f.triBase = tb;
        f.binBase = bb;
        f.accumulate = s.accumulate;
        f.light = s.light;
        f.hasXform = s.hasXform ? 1 : 0;
        if (s.hasXform) std::memcpy(f.xform, s.xform, sizeof(f.xform));
        f.occChunk = s.occChunk;
        // the lane-per-pair schedule deals one item of 32 samples to a warp
        f.occItem = b.occVariant == 1 ? 32 : s.occItem;
        e.hBases[i] = sb;
        e.hBases[nf + i] = tb;
        e.hBases[2 * nf + i] = bb;
        sb += s.W * s.H;
        tb += (int)s.nt;
        bb += s.bins * s.bins;
    }
    const bool legacy = e.stream == nullptr || e.stream == cudaStreamLegacy || e.stream == cudaStreamPerThread;
    const bool graphable = e.useGraph && !e.profile && !e.debug && !legacy;
    if (graphable) {
        GraphKey k;
        k.nf = nf;
        k.S = (int)S;
        k.T = (int)T;
        k.NB = (int)NB;
        k.P = (int)e.pairCapacity;
        k.sp = b.samplePasses;
        k.pp = b.pairPasses + 16 * b.pairTriBits;
        k.db = b.depthBits;
        k.maxS = maxS;
        k.maxT = maxT;
        k.maxV = maxV;
        k.arena = e.arena;
        k.hFrames = e.hFrames;
        k.ov = b.occVariant + 16 * b.rayCast + 32 * b.wide + 64 * e.depthPlane + 128 * b.openBox + 256 * b.rows16;
        k.stream = e.stream;
        FDZB_CUDA(refresh_lookback(e));
        if (!e.graph || !(k == e.graphKey)) {
            drop_graph(e);
            FDZB_CUDA(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t body = enqueue_body(e, nf);
            cudaGraph_t g = nullptr;
            cudaError_t end = cudaStreamEndCapture(e.stream, &g);
            if (body != cudaSuccess || end != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                return fail(FDZB_ERR_CUDA, std::string("graph capture: ") +
                                               cudaGetErrorString(body != cudaSuccess ? body : end));
            }
            cudaError_t inst = cudaGraphInstantiate(&e.graph, g, 0);
            cudaGraphDestroy(g);
            if (inst != cudaSuccess) {
                e.graph = nullptr;
                return fail(FDZB_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(inst));
            }
            e.graphKey = k;
            ++e.graphCaptures;
        } else {
            ++e.graphReplays;
        }
        FDZB_CUDA(cudaEventRecord(e.ev0, e.stream));
        FDZB_CUDA(cudaGraphLaunch(e.graph, e.stream));
        FDZB_CUDA(cudaEventRecord(e.ev1, e.stream));
        e.lastFromGraph = true;
    } else {
        FDZB_CUDA(refresh_lookback(e));
        FDZB_CUDA(cudaEventRecord(e.ev0, e.stream));
        FDZB_CUDA(enqueue_body(e, nf));
        FDZB_CUDA(cudaEventRecord(e.ev1, e.stream));
        e.lastFromGraph = false;
    }
    e.pending = true;
    return FDZB_OK;
}

namespace {

// A frame whose triangle/bin pairs do not fit the largest pair buffer runs in
// passes over ranges of its triangles, each OR-ing its occlusion bits into the
// frame's masks.  The mask is the OR over triangles, so the passes add up to
// the single-launch result; a launch whose pair list overflowed contributed a
// subset of its bits, so a range that still overflows is split in two and run
// again without undoing anything.  The far plane, light plane and bins depend
// on the samples and on all vertices, not on the triangle range, and are the
// same in every pass.
decltype(Engine::passKey) pass_key(const Engine &e, const FrameSpec &f)
{
    return {f.pos, f.nrm, f.W, f.H, f.vtx, f.idx, f.nt, f.bins, f.light.N * 128 + f.light.NC, e.maxPairCapacity};
}

int run_triangle_passes(Engine &e, bool planned)
{
    const FrameSpec full = e.frames[0];
    const size_t S = (size_t)full.W * full.H;
    const size_t words = (size_t)(full.light.N * full.light.NC + 31) / 32;
    uint32_t *masks = full.masks;
    // after an overflowed launch, full.masks already holds a subset of the bits
    int acc = planned ? 0 : 1;
    if (!masks) {
        const size_t bytes = S * words * 4;
        if (e.passMasksBytes < bytes) {
            if (e.passMasks) cudaFree(e.passMasks);
            e.passMasks = nullptr;
            e.passMasksBytes = 0;
            if (cudaMalloc(&e.passMasks, bytes) != cudaSuccess) {
                cudaGetLastError();
                return fail(FDZB_ERR_NO_MEMORY, "mask buffer for triangle passes");
            }
            e.passMasksBytes = bytes;
        }
        masks = e.passMasks;
        acc = 0;
    }
    const bool savedGraph = e.useGraph;
    e.useGraph = false;
    e.pairCapacity = e.maxPairCapacity;
    const long long T = (long long)full.nt;
    std::vector<std::pair<long long, long long>> todo;   // stack of [t0, t1), first range on top
    if (planned) {
        for (size_t i = e.passPlan.size(); i-- > 0;) todo.push_back(e.passPlan[i]);
    } else {
        const long long est = std::max<long long>((long long)e.hCounters->pairCount, e.maxPairCapacity);
        long long K = std::max<long long>(2, (est + e.maxPairCapacity * 3 / 4 - 1) / (e.maxPairCapacity * 3 / 4));
        K = std::min(K, std::max(T, 1ll));
        for (long long i = K; i-- > 0;) todo.push_back({T * i / K, T * (i + 1) / K});
    }
    std::vector<std::pair<long long, long long>> done;
    int splits = planned ? 0 : 1;   // the overflowed first launch counts as one re-plan
    e.passes = 0;
    e.passPairs = e.passTests = e.passRows = e.passPartial = 0;
    e.passValidTris = 0;
    for (float &t : e.passStageMs) t = 0.f;
    float msSum = 0.f;
    int rc = FDZB_OK;
    while (!todo.empty() && rc == FDZB_OK) {
        const auto r = todo.back();
        todo.pop_back();
        if (r.second <= r.first) continue;
        FrameSpec f = full;
        f.idx = full.idx + 3 * r.first;
        f.nt = (size_t)(r.second - r.first);
        f.masks = masks;
        f.accumulate = acc;
        e.frames.assign(1, f);
        rc = engine_enqueue(e);
        if (rc) break;
        cudaError_t w = cudaStreamSynchronize(e.stream);
        e.pending = false;
        if (w != cudaSuccess) {
            rc = fail(FDZB_ERR_CUDA, std::string("cudaStreamSynchronize: ") + cudaGetErrorString(w));
            break;
        }
        acc = 1;
        const fdzb::Counters &k = *e.hCounters;
        if (k.errorFlags) {
            rc = fail(k.errorFlags & fdzb::ERR_BAD_INPUT ? FDZB_ERR_INVALID_ARG : FDZB_ERR_DEVICE_TIMEOUT,
                      "device error during a triangle pass");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e.ev0, e.ev1);
        msSum += ms;
        ++e.passes;
        if (e.profile)
            for (int j = 0; j < fdzb::STAGE_COUNT; ++j) {
                float t = 0.f;
                cudaEventElapsedTime(&t, e.stageEv[j], e.stageEv[j + 1]);
                e.passStageMs[j] += t;
            }
        if (k.pairOverflow) {
            if (r.second - r.first <= 1) {
                rc = fail(FDZB_ERR_CAPACITY, "one triangle overflows the pair buffer");
                break;
            }
            const long long mid = (r.first + r.second) / 2;
            todo.push_back({mid, r.second});
            todo.push_back({r.first, mid});
            ++splits;
            continue;
        }
        done.push_back(r);
        e.passPairs += (unsigned long long)k.pairCount;
        e.passTests += k.pairTests;
        e.passRows += k.rowsEvaluated;
        e.passPartial += k.partialMasks;
        e.passValidTris += e.hStates[0].state == 2 ? e.hStates[0].nValidTris : 0;
    }
    e.frames.assign(1, full);
    e.useGraph = savedGraph;
    e.lastMs = msSum;
    e.replans = splits;
    if (rc == FDZB_OK) {
        e.passPlan = done;
        e.passKey = pass_key(e, full);
    } else {
        e.passPlan.clear();
    }
    return rc;
}

}  // namespace

int engine_sync(Engine &e)
{
    if (!e.pending) return FDZB_OK;
    e.replans = 0;
    for (;;) {
        // the launch's own end event, not the whole stream: work another
        // context or the caller queued behind this launch is not waited for
        cudaError_t w = cudaEventSynchronize(e.ev1);
        e.pending = false;
        if (w != cudaSuccess) return fail(FDZB_ERR_CUDA, std::string("cudaEventSynchronize: ") + cudaGetErrorString(w));
        const fdzb::Counters &k = *e.hCounters;
        if (k.errorFlags & fdzb::ERR_LOOKBACK_TIMEOUT)
            return fail(FDZB_ERR_DEVICE_TIMEOUT, "a look-back wait exceeded its spin limit");
        if (k.errorFlags & fdzb::ERR_MBAR_TIMEOUT)
            return fail(FDZB_ERR_DEVICE_TIMEOUT, "a shared-memory barrier wait exceeded its limit");
        if (k.errorFlags & fdzb::ERR_BAD_INPUT)
            return fail(FDZB_ERR_INVALID_ARG, "triangle index out of range of the vertex buffer");
        if (k.errorFlags & fdzb::ERR_INTERNAL)
            return fail(FDZB_ERR_CUDA, "internal consistency check failed on the device");
        if (!k.pairOverflow) break;
        if ((long long)k.pairCount > e.maxPairCapacity || e.pairCapacity >= e.maxPairCapacity || e.replans >= 3) {
            if (e.frames.size() == 1) return run_triangle_passes(e, false);
            return fail(FDZB_ERR_CAPACITY, "triangle/bin pair buffer overflow (" + std::to_string(k.pairCount) +
                                               " pairs) in a launch of several frames");
        }
        e.pairCapacity = std::min<long long>((long long)k.pairCount + k.pairCount / 4 + 1024, e.maxPairCapacity);
        ++e.replans;
        const int replans = e.replans;
        if (int rc = engine_enqueue(e)) return rc;
        e.replans = replans;
    }
    float ms = 0.f;
    FDZB_CUDA(cudaEventElapsedTime(&ms, e.ev0, e.ev1));
    e.lastMs = ms;
    e.passes = 1;
    if (e.lastOpenBox && e.openBoxMode == FDZB_OPEN_BOX_AUTO && !e.openBoxKeep.count(e.lastShape)) {
        const fdzb::Counters &k = *e.hCounters;
        const double rate = k.pairsExamined ? (double)k.boxSkips / (double)k.pairsExamined : 0.0;
        e.openBoxKeep[e.lastShape] = rate >= kOpenBoxKeep;
    }
    return FDZB_OK;
}

int engine_launch(Engine &e)
{
    if (e.frames.size() == 1 && !e.passPlan.empty() && e.passKey == pass_key(e, e.frames[0])) {
        const int rc = run_triangle_passes(e, true);
        e.pending = false;
        return rc;
    }
    e.passes = 1;
    return engine_enqueue(e);
}

// Statistics of frame i of the last completed launch.
void frame_stats(const Engine &e, int i, fdzb_frame_stats &o)
{
    const fdzb::FrameState &s = e.hStates[i];
    const fdzb::Counters &k = *e.hCounters;
    const FrameSpec &f = e.frames[i];
    const bool single = e.frames.size() == 1;
    std::memset(&o, 0, sizeof(o));
    o.state = (s.state == 2 && s.nValidTris == 0) ? 1 : s.state;
    o.valid_samples = o.state == 2 ? s.nValidSamples : 0;
    o.valid_triangles = s.state == 2 ? s.nValidTris : 0;
    // launch-wide counters: per frame only when the launch holds one frame
    o.num_pairs = single ? (o.state == 2 ? k.pairCount : 0) : -1;
    o.num_bins = f.bins * f.bins;
    o.pair_capacity = (int)e.pairCapacity;
    o.pair_tests = single ? (int64_t)k.pairTests : -1;
    o.f = s.f;
    o.sub[0] = s.subx;
    o.sub[1] = s.suby;
    o.lp_begin[0] = s.Bx; o.lp_begin[1] = s.By; o.lp_begin[2] = s.Bz;
    o.lp_end[0] = s.Ex; o.lp_end[1] = s.Ey; o.lp_end[2] = s.Ez;
    o.lp_factor[0] = s.fx; o.lp_factor[1] = s.fy;
    for (int j = 0; j < 6; ++j) {
        o.sample_aabb[j] = s.sampleAabb[j];
        o.model_aabb[j] = s.modelAabb[j];
    }
    o.replans = e.replans;
    o.quirk_key_range = s.quirkKeyRange;
    o.kernel_launches = e.launches;
    o.triangle_passes = e.passes;
    o.rows_evaluated = single ? (int64_t)k.rowsEvaluated : -1;
    o.partial_masks = single ? (int64_t)k.partialMasks : -1;
    if (single && e.passes > 1) {
        o.num_pairs = (int32_t)std::min<unsigned long long>(e.passPairs, 0x7fffffffull);
        o.pair_tests = (int64_t)e.passTests;
        o.rows_evaluated = (int64_t)e.passRows;
        o.partial_masks = (int64_t)e.passPartial;
        o.valid_triangles = o.state == 2 ? (int32_t)e.passValidTris : 0;
        o.kernel_launches = e.launches * e.passes;
    }
    for (int j = 0; j < fdzb::STAGE_COUNT; ++j) {
        float t = 0.f;
        if (e.profile) {
            if (single && e.passes > 1) t = e.passStageMs[j];
            else cudaEventElapsedTime(&t, e.stageEv[j], e.stageEv[j + 1]);
        }
        o.stage_ms[j] = t;
    }
}

void launch_stats(const Engine &e, fdzb_frame_stats &o)
{
    const fdzb::Counters &k = *e.hCounters;
    std::memset(&o, 0, sizeof(o));
    o.state = 2;
    long long vs = 0, vt = 0, nb = 0;
    for (size_t i = 0; i < e.frames.size(); ++i) {
        const fdzb::FrameState &s = e.hStates[i];
        if (s.state == 2 && s.nValidTris > 0) {
            vs += s.nValidSamples;
            vt += s.nValidTris;
        }
        o.quirk_key_range += s.quirkKeyRange;
        nb += (long long)e.frames[i].bins * e.frames[i].bins;
    }
    o.valid_samples = (int32_t)std::min<long long>(vs, 0x7fffffff);
    o.valid_triangles = (int32_t)std::min<long long>(vt, 0x7fffffff);
    o.num_pairs = k.pairCount;
    o.num_bins = (int32_t)nb;
    o.pair_capacity = (int)e.pairCapacity;
    o.pair_tests = (int64_t)k.pairTests;
    o.replans = e.replans;
    o.kernel_launches = e.launches;
    o.rows_evaluated = (int64_t)k.rowsEvaluated;
    o.partial_masks = (int64_t)k.partialMasks;
    for (int j = 0; j < fdzb::STAGE_COUNT; ++j) {
        float t = 0.f;
        if (e.profile) cudaEventElapsedTime(&t, e.stageEv[j], e.stageEv[j + 1]);
        o.stage_ms[j] = t;
    }
}

}  // namespace fdzb

using namespace fdzb;


// ---- FD-shaped context: one scene, one view, one light -----------------------

struct fdzb_ctx {
    Engine eng;
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
    fdzb_frame_stats stats{};
    bool hasXform = false;
    float xform[16] = {};
    int occChunk = 32, occItem = 32;   // occlusion shape (fdzb_ctx_set_occlusion_shape)
};

// ---- batch: a list of independent frames per launch --------------------------

struct fdzb_batch {
    Engine eng;
    int triOrder = FDZB_TRI_ORDER_COVERAGE;
    TuneTable tuned;
    std::vector<TuneChoice> chosen;
    long long tuneLaunches = 0;
    int occChunk = 0, occItem = 0;   // a shape set for every frame (0: tuned or default)
};

namespace {

int ctx_check(fdzb_ctx *c)
{
    if (!c) return fail(FDZB_ERR_NOT_INITIALIZED, "context not initialised (call fdzb_init)");
    return FDZB_OK;
}

int batch_check(fdzb_batch *b)
{
    if (!b) return fail(FDZB_ERR_NOT_INITIALIZED, "batch is NULL");
    return FDZB_OK;
}

int ctx_frame(fdzb_ctx *c, FrameSpec &f)
{
    if (c->W <= 0 || c->H <= 0) return fail(FDZB_ERR_NOT_READY, "view size not set (fdzb_set_view)");
    if (!c->pos || !c->nrm) return fail(FDZB_ERR_NOT_READY, "sample buffers not set");
    if (!c->shadow) return fail(FDZB_ERR_NOT_READY, "output buffer not set");
    if (c->models.empty()) return fail(FDZB_ERR_NOT_READY, "no model added");
    if (!c->lightSet) return fail(FDZB_ERR_NOT_READY, "area light not set");
    const Model &m = c->models[0];  // only scene 0 / model 0 is drawn (FS/api.cpp:430-445)
    f.pos = c->pos;
    f.nrm = c->nrm;
    f.W = c->W;
    f.H = c->H;
    f.vtx = m.vtx;
    f.nv = m.nv;
    f.strideBytes = m.strideBytes;
    f.idx = m.idx;
    f.nt = m.nt;
    f.light = c->light;
    f.bins = c->bins;
    f.cull = c->cull;
    f.esp = c->esp;
    f.shadow = c->shadow;
    f.masks = c->masks;
    f.hasXform = c->hasXform;
    if (c->hasXform) std::memcpy(f.xform, c->xform, sizeof(f.xform));
    f.occChunk = c->occChunk;
    f.occItem = c->occItem;
    return FDZB_OK;
}

int ctx_sync(fdzb_ctx *c)
{
    if (!c->eng.pending) return FDZB_OK;
    if (int rc = engine_sync(c->eng)) return rc;
    frame_stats(c->eng, 0, c->stats);
    return FDZB_OK;
}

// A frame without a bin grid takes its class's tuned grid and shape; a shape set
// on the batch applies to every frame.
void batch_shape_for(fdzb_batch *b, FrameSpec &f)
{
    if (f.bins == 0) {
        const TuneChoice c = tuned_shape(b->tuned, f);
        f.bins = c.bins;
        f.occChunk = c.chunk;
        f.occItem = c.item;
    }
    if (b->occChunk) f.occChunk = b->occChunk;
    if (b->occItem) f.occItem = b->occItem;
}

}  // namespace

int fdzb::set_error(int code, const std::string &msg) { return fail(code, msg); }

// Starting point of the autotuner: about 128 samples per bin on the light plane
// (the HD frame's 1920x1080 samples over 128 x 128 bins), clamped to [8, 256].
int fdzb::heuristic_bins(long long S)
{
    const double side = std::sqrt((double)std::max(S, 1ll) / 128.0);
    int b = 8;
    while (b < 256 && b * 2 <= side * 1.41421356) b *= 2;
    return b;
}

int fdzb::desc_to_spec(const fdzb_frame_desc &d, FrameSpec &f, int i)
{
    const fdzb_area_light_desc &L = d.light;
    if (L.lightResWidth < 1 || L.lightResWidth > fdzb::kMaxLightN || L.lightResHeight < 1 ||
        L.lightResHeight > fdzb::kMaxLightN)
        return fail(FDZB_ERR_UNSUPPORTED, "frame " + std::to_string(i) + ": light grid width and height must be in [1, 64]");
    f.pos = (const float4 *)d.d_pos;
    f.nrm = (const float4 *)d.d_nrm;
    f.W = d.W;
    f.H = d.H;
    f.vtx = d.d_vtx;
    f.nv = d.n_vtx;
    f.strideBytes = d.vtx_stride_bytes;
    f.idx = d.d_idx;
    f.nt = d.n_tri;
    fdzb::light_setup(L.rightRadius, L.topRadius, L.position, L.viewDir, L.upDir, L.lightResWidth,
                      L.lightResHeight, &f.light);
    f.bins = d.bins;
    f.cull = d.cull;
    f.esp = d.esp;
    f.shadow = d.d_shadow;
    f.masks = d.d_masks;
    f.hasXform = d.model_transform != nullptr;
    if (f.hasXform) std::memcpy(f.xform, d.model_transform, sizeof(f.xform));
    return FDZB_OK;
}

size_t fdzb::launch_bytes(const std::vector<FrameSpec> &frames, long long pairCapacity, bool debug)
{
    long long S = 0, T = 0, NB = 0;
    for (const FrameSpec &f : frames) {
        S += (long long)f.W * f.H;
        T += (long long)f.nt;
        NB += (long long)f.bins * f.bins;
    }
    DeviceBuffers probe{};
    return layout(probe, nullptr, (int)frames.size(), S, T, NB, pairCapacity, debug);
}

long long fdzb::default_pair_capacity(long long T)
{
    return std::min(std::max<long long>(1 << 20, T * 64), kMaxPairCapacity);
}

fdzb::TuneKey fdzb::tune_key(long long S, long long T, int N)
{
    return TuneKey(ceil_log2(std::max(S, 1ll)), ceil_log2(std::max(T, 1ll)), N);
}

fdzb::TuneChoice fdzb::tuned_shape(const TuneTable &table, const FrameSpec &f)
{
    const long long S = (long long)f.W * f.H;
    auto it = table.find(tune_key(S, (long long)f.nt, f.light.N * 128 + f.light.NC));
    if (it != table.end()) return it->second;
    TuneChoice c;
    c.bins = heuristic_bins(S);
    return c;
}

bool fdzb::valid_occ_shape(int chunk, int item)
{
    return (chunk == 8 || chunk == 16 || chunk == 32) && (item == 32 || item == 64 || item == 128);
}

// For every size class of `frames` not in `table`, three steps, each candidate
// timed as a launch of up to 8 copies of the class's first frame (shadows into
// `scratch`, no masks) so that the GPU is as full as inside a batch, twice,
// the faster of the two counting: the grids h/2, h, 2h around the heuristic h
// (32 staged triangles, items of 32 samples); then, at the best grid, staging
// chunks of 16; then, at the best grid and chunk, items of 64 samples (half as
// many warps per bin).  Each step keeps a candidate only if it is faster.
int fdzb::autotune_bins(Engine &e, TuneTable &table, const std::vector<FrameSpec> &frames, float *scratch,
                        size_t scratchFloats, long long *launches)
{
    if (!scratch) return fail(FDZB_ERR_INVALID_ARG, "scratch buffer is NULL");
    std::map<TuneKey, size_t> firstOf;
    for (size_t i = 0; i < frames.size(); ++i) {
        const FrameSpec &f = frames[i];
        const TuneKey k = tune_key((long long)f.W * f.H, (long long)f.nt, f.light.N * 128 + f.light.NC);
        if (!table.count(k) && !firstOf.count(k)) firstOf[k] = i;
    }
    const bool savedGraph = e.useGraph;
    e.useGraph = false;  // one-off shapes: no point capturing them
    int rc = FDZB_OK;
    for (const auto &kv : firstOf) {
        const FrameSpec &f = frames[kv.second];
        const long long S = (long long)f.W * f.H;
        if ((size_t)S > scratchFloats) {
            rc = fail(FDZB_ERR_INVALID_ARG, "autotune scratch smaller than a frame");
            break;
        }
        // copies: up to 8, ~2M samples and ~1M triangles in all, within the scratch
        const long long T = std::max<long long>((long long)f.nt, 1);
        const int reps = (int)std::max(1ll, std::min<long long>({8, (2'000'000 + S - 1) / S, 1'000'000 / T,
                                                                 (long long)(scratchFloats / S)}));
        const int h = heuristic_bins(S);
        TuneChoice best;
        best.bins = h;
        float bestMs = 1e30f;
        std::vector<TuneChoice> cands;
        auto timeit = [&](const TuneChoice &c) -> float {
            std::vector<FrameSpec> specs((size_t)reps, f);
            for (int r = 0; r < reps; ++r) {
                specs[r].bins = c.bins;
                specs[r].occChunk = c.chunk;
                specs[r].occItem = c.item;
                specs[r].shadow = scratch + (size_t)r * S;
                specs[r].masks = nullptr;
            }
            float t = 1e30f;
            for (int trial = 0; trial < 2 && rc == FDZB_OK; ++trial) {
                e.frames = specs;
                rc = engine_enqueue(e);
                if (rc == FDZB_OK) rc = engine_sync(e);
                if (launches) ++*launches;
                if (rc == FDZB_OK) t = std::min(t, e.lastMs);
            }
            if (rc == FDZB_ERR_CAPACITY) {   // too many pairs at this grid: not a candidate
                rc = FDZB_OK;
                return 1e30f;
            }
            return t;
        };
        for (int cand : {h / 2, h, h * 2}) {
            if (cand < 4 || cand > kMaxBins) continue;
            TuneChoice c;
            c.bins = cand;
            const float t = timeit(c);
            if (rc) break;
            if (t < bestMs) {
                bestMs = t;
                best = c;
            }
        }
        for (int step = 0; step < 2 && rc == FDZB_OK && bestMs < 1e30f; ++step) {
            TuneChoice c = best;
            if (step == 0) c.chunk = 16;
            else c.item = 64;
            const float t = timeit(c);
            if (rc) break;
            if (t < bestMs) {
                bestMs = t;
                best = c;
            }
        }
        if (rc) break;
        table[kv.first] = best;
    }
    e.useGraph = savedGraph;
    return rc;
}


namespace {
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

extern "C" {

const char *fdzb_last_error(void) { return g_err.c_str(); }
const char *fdzb_version(void) { return "fdzb-b200 0.2 (sm_100a)"; }

int fdzb_ctx_create(fdzb_ctx **out, int device)
{
    if (!out) return fail(FDZB_ERR_INVALID_ARG, "out is NULL");
    fdzb_ctx *c = new (std::nothrow) fdzb_ctx();
    if (!c) return fail(FDZB_ERR_NO_MEMORY, "host allocation failed");
    int rc = engine_init(c->eng, device);
    if (rc) {
        engine_release(c->eng);
        delete c;
        return rc;
    }
    *out = c;
    return FDZB_OK;
}

int fdzb_ctx_destroy(fdzb_ctx *c)
{
    if (!c) return FDZB_OK;
    engine_release(c->eng);
    delete c;
    return FDZB_OK;
}

int fdzb_ctx_set_stream(fdzb_ctx *c, void *stream)
{
    if (int rc = ctx_check(c)) return rc;
    if (int rc = ctx_sync(c)) return rc;
    c->eng.stream = stream ? (cudaStream_t)stream : c->eng.ownStream;
    return FDZB_OK;
}

int fdzb_ctx_set_debug(fdzb_ctx *c, int flags)
{
    if (int rc = ctx_check(c)) return rc;
    c->eng.debug = flags & 1;
    c->eng.separatePairs = (flags & 2) != 0;
    return FDZB_OK;
}

int fdzb_ctx_set_profiling(fdzb_ctx *c, int enable)
{
    if (int rc = ctx_check(c)) return rc;
    if (enable < 0 || enable > FDZB_PROFILE_STAGES) return fail(FDZB_ERR_INVALID_ARG, "profiling mode must be 0, 1 or 2");
    c->eng.profile = enable != 0;
    c->eng.countWork = enable == FDZB_PROFILE_ALL;
    return FDZB_OK;
}

int fdzb_ctx_set_graph(fdzb_ctx *c, int enable)
{
    if (int rc = ctx_check(c)) return rc;
    if (int rc = ctx_sync(c)) return rc;
    c->eng.useGraph = enable != 0;
    if (!c->eng.useGraph) drop_graph(c->eng);
    return FDZB_OK;
}

int fdzb_ctx_set_launch_epoch(fdzb_ctx *c, uint32_t value)
{
    if (int rc = ctx_check(c)) return rc;
    if (!c->eng.arena) return fail(FDZB_ERR_NOT_READY, "no launch yet");
    if (value >= kEpochLimit) return fail(FDZB_ERR_INVALID_ARG, "epoch must be below FDZB_LOOKBACK_EPOCH_LIMIT");
    if (int rc = ctx_sync(c)) return rc;
    FDZB_CUDA(cudaMemcpyAsync(c->eng.buf.epochWord, &value, sizeof(value), cudaMemcpyHostToDevice, c->eng.stream));
    FDZB_CUDA(cudaStreamSynchronize(c->eng.stream));
    c->eng.epochCount = value;
    return FDZB_OK;
}

int fdzb_ctx_get_launch_epoch(fdzb_ctx *c, uint32_t *out)
{
    if (int rc = ctx_check(c)) return rc;
    if (!out) return fail(FDZB_ERR_INVALID_ARG, "out is NULL");
    if (!c->eng.arena) return fail(FDZB_ERR_NOT_READY, "no launch yet");
    if (int rc = ctx_sync(c)) return rc;
    FDZB_CUDA(cudaMemcpy(out, c->eng.buf.epochWord, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return FDZB_OK;
}

int fdzb_measure_alu_rate(double *lane_ops_per_second)
{
    if (!lane_ops_per_second) return fail(FDZB_ERR_INVALID_ARG, "out is NULL");
    FDZB_CUDA(fdzb::measure_alu_rate(lane_ops_per_second));
    return FDZB_OK;
}

int fdzb_check_division(uint64_t trials, uint64_t seed, uint64_t *mismatches, uint64_t *checked)
{
    if (!mismatches || !checked) return fail(FDZB_ERR_INVALID_ARG, "out is NULL");
    unsigned long long m = 0, n = 0;
    FDZB_CUDA(fdzb::check_division(trials, seed, &m, &n));
    *mismatches = m;
    *checked = n;
    return FDZB_OK;
}

int fdzb_ctx_set_open_box(fdzb_ctx *c, int mode)
{
    if (int rc = ctx_check(c)) return rc;
    if (mode != FDZB_OPEN_BOX_OFF && mode != FDZB_OPEN_BOX_ON && mode != FDZB_OPEN_BOX_AUTO)
        return fail(FDZB_ERR_INVALID_ARG, "open-box mode: FDZB_OPEN_BOX_OFF, _ON or _AUTO");
    if (int rc = ctx_sync(c)) return rc;
    c->eng.openBoxMode = mode;
    c->eng.openBoxKeep.clear();
    return FDZB_OK;
}

int fdzb_batch_set_open_box(fdzb_batch *b, int mode)
{
    if (int rc = batch_check(b)) return rc;
    if (mode != FDZB_OPEN_BOX_OFF && mode != FDZB_OPEN_BOX_ON && mode != FDZB_OPEN_BOX_AUTO)
        return fail(FDZB_ERR_INVALID_ARG, "open-box mode: FDZB_OPEN_BOX_OFF, _ON or _AUTO");
    if (int rc = engine_sync(b->eng)) return rc;
    b->eng.openBoxMode = mode;
    b->eng.openBoxKeep.clear();
    return FDZB_OK;
}

int fdzb_ctx_set_occlusion_shape(fdzb_ctx *c, int chunk, int item)
{
    if (int rc = ctx_check(c)) return rc;
    if (!valid_occ_shape(chunk, item))
        return fail(FDZB_ERR_INVALID_ARG, "occlusion shape: chunk in {8, 16, 32}, item in {32, 64, 128}");
    c->occChunk = chunk;
    c->occItem = item;
    return FDZB_OK;
}

int fdzb_ctx_set_occlusion_schedule(fdzb_ctx *c, int schedule)
{
    if (int rc = ctx_check(c)) return rc;
    if (schedule != FDZB_OCC_LANE_PER_SAMPLE && schedule != FDZB_OCC_LANE_PER_PAIR)
        return fail(FDZB_ERR_INVALID_ARG, "unknown occlusion schedule");
    c->eng.occVariant = schedule;
    return FDZB_OK;
}

int fdzb_ctx_set_pair_capacity_limit(fdzb_ctx *c, int64_t pairs)
{
    if (int rc = ctx_check(c)) return rc;
    if (int rc = ctx_sync(c)) return rc;
    if (pairs < 1024 || pairs > kMaxPairCapacity)
        return fail(FDZB_ERR_INVALID_ARG, "pair capacity limit must be in [1024, 2^29]");
    c->eng.maxPairCapacity = pairs;
    c->eng.pairCapacity = std::min<long long>(c->eng.pairCapacity, pairs);
    return FDZB_OK;
}

int fdzb_ctx_set_tri_order(fdzb_ctx *c, int order)
{
    if (int rc = ctx_check(c)) return rc;
    if (order != FDZB_TRI_ORDER_REFERENCE && order != FDZB_TRI_ORDER_COVERAGE)
        return fail(FDZB_ERR_INVALID_ARG, "unknown triangle order");
    c->eng.triOrder = order;
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
    if (d->lightResWidth < 1 || d->lightResWidth > fdzb::kMaxLightN || d->lightResHeight < 1 ||
        d->lightResHeight > fdzb::kMaxLightN)
        return fail(FDZB_ERR_UNSUPPORTED, "light grid width and height must be in [1, 64]");
    c->lightDesc = *d;
    fdzb::light_setup(d->rightRadius, d->topRadius, d->position, d->viewDir, d->upDir, d->lightResWidth,
                      d->lightResHeight, &c->light);
    c->lightSet = true;
    return FDZB_OK;
}

int fdzb_ctx_set_shadow_method(fdzb_ctx *c, int method)
{
    if (int rc = ctx_check(c)) return rc;
    if (method != FDZB_SHADOW_EDGE_MASKS && method != FDZB_SHADOW_RAY_CAST)
        return fail(FDZB_ERR_INVALID_ARG, "unknown shadow method");
    if (int rc = ctx_sync(c)) return rc;
    c->eng.rayCast = method == FDZB_SHADOW_RAY_CAST ? 1 : 0;
    return FDZB_OK;
}

int fdzb_ctx_set_depth_plane(fdzb_ctx *c, int enable)
{
    if (int rc = ctx_check(c)) return rc;
    if (int rc = ctx_sync(c)) return rc;
    c->eng.depthPlane = enable ? 1 : 0;
    return FDZB_OK;
}

int fdzb_ctx_set_model_transform(fdzb_ctx *c, const float m[16])
{
    if (int rc = ctx_check(c)) return rc;
    c->hasXform = m != nullptr;
    if (m) std::memcpy(c->xform, m, sizeof(c->xform));
    return FDZB_OK;
}

int fdzb_ctx_move_model(fdzb_ctx *c, const float m[16])
{
    if (int rc = ctx_check(c)) return rc;
    if (!m) return fail(FDZB_ERR_INVALID_ARG, "matrix is NULL");
    if (c->models.empty()) return fail(FDZB_ERR_NOT_READY, "no model added");
    if (int rc = ctx_sync(c)) return rc;
    const Model &md = c->models[0];
    FDZB_CUDA(fdzb::run_move_model(const_cast<float *>(md.vtx), (int)(md.strideBytes / 4), (int)md.nv, m,
                                   c->eng.stream));
    FDZB_CUDA(cudaStreamSynchronize(c->eng.stream));
    return FDZB_OK;
}

int fdzb_ctx_launch_async(fdzb_ctx *c)
{
    if (int rc = ctx_check(c)) return rc;
    if (int rc = ctx_sync(c)) return rc;
    FrameSpec f;
    if (int rc = ctx_frame(c, f)) return rc;
    c->eng.frames.assign(1, f);
    const int rc = engine_launch(c->eng);
    if (rc == FDZB_OK && !c->eng.pending) frame_stats(c->eng, 0, c->stats);
    return rc;
}

int fdzb_ctx_sync(fdzb_ctx *c)
{
    if (int rc = ctx_check(c)) return rc;
    return ctx_sync(c);
}

int fdzb_ctx_launch(fdzb_ctx *c, float *ms)
{
    int rc = fdzb_ctx_launch_async(c);
    if (rc) return rc;
    rc = ctx_sync(c);
    if (rc) return rc;
    if (ms) *ms = c->eng.lastMs;
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
    if (!c->eng.arena) return fail(FDZB_ERR_NOT_READY, "no launch yet");
    if (int rc = ctx_sync(c)) return rc;
    const fdzb::DeviceBuffers &b = c->eng.buf;
    const size_t S = (size_t)b.totalSamples, T = (size_t)b.totalTris, NB = (size_t)b.totalBins;
    const size_t P = (size_t)std::min(c->eng.hCounters->pairCount, b.pairCapacity);
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
    case FDZB_ARR_SORTED_PAIR_BIN:
    case FDZB_ARR_PAIR_TRI:
    case FDZB_ARR_SORTED_PAIR_TRI: {
        // pair keys are the global bins, values the triangles -- or one word
        // bin << pairTriBits | triangle each
        const bool pre = what == FDZB_ARR_PAIR_BIN || what == FDZB_ARR_PAIR_TRI;
        const bool wantBin = what == FDZB_ARR_PAIR_BIN || what == FDZB_ARR_SORTED_PAIR_BIN;
        const int tb = b.pairTriBits;
        const uint32_t *s2 = nullptr;
        if (tb || wantBin) s2 = pre ? b.dbgPKeys : (pOdd ? b.pkeysB : b.pkeysA);
        else s2 = pre ? b.dbgPVals : (pOdd ? b.pvalsB : b.pvalsA);
        if (!s2) return fail(FDZB_ERR_NOT_READY, "pre-sort arrays need fdzb_ctx_set_debug(ctx, 1)");
        if (bytes > 4 * P) return fail(FDZB_ERR_INVALID_ARG, "export size exceeds the array");
        if (!bytes) return FDZB_OK;
        FDZB_CUDA(cudaMemcpy(dst, s2, bytes, cudaMemcpyDeviceToHost));
        if (tb) {
            uint32_t *o = (uint32_t *)dst;
            const uint32_t mask = (1u << tb) - 1u;
            for (size_t i = 0; i < bytes / 4; ++i) o[i] = wantBin ? (o[i] >> tb) : (o[i] & mask);
        }
        return FDZB_OK;
    }
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
    case FDZB_ARR_WORK_COUNTERS: {
        const fdzb::Counters &k = *c->eng.hCounters;
        const uint64_t v[7] = {k.pairTests, k.rowsEvaluated, k.partialMasks, k.pairsExamined, k.chunks, k.rounds,
                               k.boxSkips};
        if (bytes > sizeof(v)) return fail(FDZB_ERR_INVALID_ARG, "export size exceeds the array");
        std::memcpy(dst, v, bytes);
        return FDZB_OK;
    }
    default: return fail(FDZB_ERR_INVALID_ARG, "unknown array id");
    }
    if (bytes > avail) return fail(FDZB_ERR_INVALID_ARG, "export size exceeds the array");
    if (bytes) FDZB_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return FDZB_OK;
}

int fdzb_light_sample_positions(const fdzb_area_light_desc *d, float *out)
{
    if (!d || !out) return fail(FDZB_ERR_INVALID_ARG, "NULL argument");
    if (d->lightResWidth < 1 || d->lightResHeight < 1 || d->lightResWidth > 64 || d->lightResHeight > 64)
        return fail(FDZB_ERR_INVALID_ARG, "bad light grid");
    fdzb::LightParams L;
    fdzb::light_setup(d->rightRadius, d->topRadius, d->position, d->viewDir, d->upDir, d->lightResWidth,
                      d->lightResHeight, &L);
    for (int i = 0; i < d->lightResHeight; ++i)
        for (int j = 0; j < d->lightResWidth; ++j) {
            float *p = out + 3 * (i * d->lightResWidth + j);
            for (int k = 0; k < 3; ++k) {
                const float a = L.ur[k] + L.xd[k] * (float)j;   // (upRight + x_delt*j) + y_delt*i
                p[k] = a + L.yd[k] * (float)i;
            }
        }
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

// ---- batches -----------------------------------------------------------------

int fdzb_batch_create(fdzb_batch **out, int device)
{
    if (!out) return fail(FDZB_ERR_INVALID_ARG, "out is NULL");
    fdzb_batch *b = new (std::nothrow) fdzb_batch();
    if (!b) return fail(FDZB_ERR_NO_MEMORY, "host allocation failed");
    int rc = engine_init(b->eng, device);
    if (rc) {
        engine_release(b->eng);
        delete b;
        return rc;
    }
    *out = b;
    return FDZB_OK;
}

int fdzb_batch_destroy(fdzb_batch *b)
{
    if (!b) return FDZB_OK;
    engine_release(b->eng);
    delete b;
    return FDZB_OK;
}

int fdzb_batch_set_stream(fdzb_batch *b, void *stream)
{
    if (int rc = batch_check(b)) return rc;
    if (int rc = engine_sync(b->eng)) return rc;
    b->eng.stream = stream ? (cudaStream_t)stream : b->eng.ownStream;
    return FDZB_OK;
}

int fdzb_batch_set_graph(fdzb_batch *b, int enable)
{
    if (int rc = batch_check(b)) return rc;
    if (int rc = engine_sync(b->eng)) return rc;
    b->eng.useGraph = enable != 0;
    if (!b->eng.useGraph) drop_graph(b->eng);
    return FDZB_OK;
}

int fdzb_batch_set_profiling(fdzb_batch *b, int enable)
{
    if (int rc = batch_check(b)) return rc;
    if (enable < 0 || enable > FDZB_PROFILE_STAGES) return fail(FDZB_ERR_INVALID_ARG, "profiling mode must be 0, 1 or 2");
    b->eng.profile = enable != 0;
    b->eng.countWork = enable == FDZB_PROFILE_ALL;
    return FDZB_OK;
}

int fdzb_batch_set_occlusion_schedule(fdzb_batch *b, int schedule)
{
    if (int rc = batch_check(b)) return rc;
    if (schedule != FDZB_OCC_LANE_PER_SAMPLE && schedule != FDZB_OCC_LANE_PER_PAIR)
        return fail(FDZB_ERR_INVALID_ARG, "unknown occlusion schedule");
    b->eng.occVariant = schedule;
    return FDZB_OK;
}

int fdzb_batch_set_depth_plane(fdzb_batch *b, int enable)
{
    if (int rc = batch_check(b)) return rc;
    b->eng.depthPlane = enable ? 1 : 0;
    return FDZB_OK;
}

int fdzb_batch_set_tri_order(fdzb_batch *b, int order)
{
    if (int rc = batch_check(b)) return rc;
    if (order != FDZB_TRI_ORDER_REFERENCE && order != FDZB_TRI_ORDER_COVERAGE)
        return fail(FDZB_ERR_INVALID_ARG, "unknown triangle order");
    b->eng.triOrder = order;
    return FDZB_OK;
}

int fdzb_batch_launch_async(fdzb_batch *b, const fdzb_frame_desc *frames, int n)
{
    if (int rc = batch_check(b)) return rc;
    if (!frames || n <= 0) return fail(FDZB_ERR_INVALID_ARG, "empty frame list");
    if (int rc = engine_sync(b->eng)) return rc;
    std::vector<FrameSpec> specs((size_t)n);
    b->chosen.assign((size_t)n, TuneChoice{});
    for (int i = 0; i < n; ++i) {
        if (int rc = desc_to_spec(frames[i], specs[i], i)) return rc;
        batch_shape_for(b, specs[i]);
        b->chosen[i].bins = specs[i].bins;
        b->chosen[i].chunk = specs[i].occChunk;
        b->chosen[i].item = specs[i].occItem;
    }
    b->eng.frames.swap(specs);
    return engine_launch(b->eng);
}

int fdzb_batch_sync(fdzb_batch *b, float *ms)
{
    if (int rc = batch_check(b)) return rc;
    if (int rc = engine_sync(b->eng)) return rc;
    if (ms) *ms = b->eng.lastMs;
    return FDZB_OK;
}

int fdzb_batch_launch(fdzb_batch *b, const fdzb_frame_desc *frames, int n, float *ms)
{
    if (int rc = fdzb_batch_launch_async(b, frames, n)) return rc;
    return fdzb_batch_sync(b, ms);
}

int fdzb_batch_get_frame_stats(fdzb_batch *b, int i, fdzb_frame_stats *out)
{
    if (int rc = batch_check(b)) return rc;
    if (!out) return fail(FDZB_ERR_INVALID_ARG, "out is NULL");
    if (b->eng.pending) return fail(FDZB_ERR_NOT_READY, "launch not synchronised (fdzb_batch_sync)");
    if (i < 0 || i >= (int)b->eng.frames.size()) return fail(FDZB_ERR_INVALID_ARG, "frame index out of range");
    frame_stats(b->eng, i, *out);
    return FDZB_OK;
}

int fdzb_batch_get_stats(fdzb_batch *b, fdzb_batch_stats *out)
{
    if (int rc = batch_check(b)) return rc;
    if (!out) return fail(FDZB_ERR_INVALID_ARG, "out is NULL");
    if (b->eng.pending) return fail(FDZB_ERR_NOT_READY, "launch not synchronised (fdzb_batch_sync)");
    std::memset(out, 0, sizeof(*out));
    launch_stats(b->eng, out->totals);
    out->frames = (int32_t)b->eng.frames.size();
    out->from_graph = b->eng.lastFromGraph ? 1 : 0;
    out->graph_captures = b->eng.graphCaptures;
    out->graph_replays = b->eng.graphReplays;
    out->tuned_classes = (int32_t)b->tuned.size();
    out->tune_launches = b->tuneLaunches;
    out->ms = b->eng.lastMs;
    return FDZB_OK;
}

int fdzb_batch_frame_bins(fdzb_batch *b, int i)
{
    if (int rc = batch_check(b)) return rc;
    if (i < 0 || i >= (int)b->chosen.size()) return fail(FDZB_ERR_INVALID_ARG, "frame index out of range");
    return b->chosen[i].bins;
}

int fdzb_batch_frame_shape(fdzb_batch *b, int i, int *bins, int *chunk, int *item)
{
    if (int rc = batch_check(b)) return rc;
    if (i < 0 || i >= (int)b->chosen.size()) return fail(FDZB_ERR_INVALID_ARG, "frame index out of range");
    if (bins) *bins = b->chosen[i].bins;
    if (chunk) *chunk = b->chosen[i].chunk;
    if (item) *item = b->chosen[i].item;
    return FDZB_OK;
}

int fdzb_batch_set_occlusion_shape(fdzb_batch *b, int chunk, int item)
{
    if (int rc = batch_check(b)) return rc;
    if ((chunk || item) && !valid_occ_shape(chunk ? chunk : 32, item ? item : 32))
        return fail(FDZB_ERR_INVALID_ARG, "occlusion shape: chunk in {8, 16, 32}, item in {32, 64, 128}");
    b->occChunk = chunk;
    b->occItem = item;
    return FDZB_OK;
}

// Times candidate bin resolutions for every size class present in `frames`
// (frames with bins == 0 only) and keeps the fastest.  Each candidate runs as a
// launch of `reps` copies of the class's first frame (so that it is timed as
// it runs inside a batch: the GPU full), writing into `d_scratch`
// (float[scratch_floats]), twice; the faster of the two counts.
int fdzb_batch_autotune(fdzb_batch *b, const fdzb_frame_desc *frames, int n, float *d_scratch,
                        size_t scratch_floats)
{
    if (int rc = batch_check(b)) return rc;
    if (!frames || n <= 0) return fail(FDZB_ERR_INVALID_ARG, "empty frame list");
    if (int rc = engine_sync(b->eng)) return rc;
    std::vector<FrameSpec> specs;
    for (int i = 0; i < n; ++i) {
        if (frames[i].bins != 0) continue;
        FrameSpec f;
        if (int rc = desc_to_spec(frames[i], f, i)) return rc;
        specs.push_back(f);
    }
    return autotune_bins(b->eng, b->tuned, specs, d_scratch, scratch_floats, &b->tuneLaunches);
}

// ---- reference-shaped global context -----------------------------------------

int fdzb_init(void)
{
    if (g_ctx) {
        fdzb_ctx_destroy(g_ctx);
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
