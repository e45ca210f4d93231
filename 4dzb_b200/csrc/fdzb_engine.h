// fdzb_engine.h -- the launch engine shared by contexts, batches and the server.
//
// An Engine owns one device arena (every scratch buffer of a launch), pinned
// staging blocks, a stream and the CUDA graph of its last launch shape.  It runs
// a list of frames (FrameSpec) through the pipeline in one launch per stage.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/fdzb.h"
#include "fdzb_internal.h"

namespace fdzb {

// Host copy of one frame's inputs.
struct FrameSpec {
    const float4 *pos = nullptr, *nrm = nullptr;
    int W = 0, H = 0;
    const float *vtx = nullptr;
    size_t nv = 0, strideBytes = 16;
    const int32_t *idx = nullptr;
    size_t nt = 0;
    LightParams light{};
    int bins = 16;
    int cull = 1;
    float esp = 1e-6f;
    float *shadow = nullptr;
    uint32_t *masks = nullptr;
    int accumulate = 0;   // OR into `masks` (a later triangle pass of the same frame)
    bool hasXform = false;  // vertices read through xform (column-major 4x4)
    float xform[16] = {};
    int occChunk = 32;      // occlusion shape (FrameDesc::occChunk, occItem)
    int occItem = 32;
};

// Host-side parameters that a captured graph bakes in; a launch whose key
// differs re-captures.
struct GraphKey {
    int nf = -1, S = 0, T = 0, NB = 0, P = 0, sp = 0, pp = 0, db = 0, maxS = 0, maxT = 0, maxV = 0;
    int ov = 0;   // occlusion kernel choice (schedule, ray cast)
    const void *arena = nullptr, *hFrames = nullptr;
    cudaStream_t stream = nullptr;
    auto tie() const
    {
        return std::tie(nf, S, T, NB, P, sp, pp, db, maxS, maxT, maxV, ov, arena, hFrames, stream);
    }
    bool operator==(const GraphKey &o) const { return tie() == o.tie(); }
};

struct Engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t ownStream = nullptr;
    void *arena = nullptr;
    size_t arenaBytes = 0;
    DeviceBuffers buf{};
    long long pairCapacity = 0;
    int debug = 0;  // keep pre-sort copies for export
    bool separatePairs = false;  // pairs as key/value arrays even where one word would hold them
    int triOrder = FDZB_TRI_ORDER_COVERAGE;
    bool profile = false;  // record events at the stage boundaries
    bool countWork = false;  // with profile: the occlusion kernel form that counts its work
    bool useGraph = true;
    int occVariant = 0;    // occlusion kernel (DeviceBuffers::occVariant)
    int rayCast = 0;       // ray-cast cross-check instead of edge masks (DeviceBuffers::rayCast)
    int depthPlane = 0;    // edge masks also test each triangle's own plane (FrameDesc::depthPlane)
    long long maxPairCapacity = 1ll << 29;   // largest pair buffer; beyond it a frame runs in triangle passes
    // triangle passes of the last single-frame launch (1 = none) and their sums
    int passes = 1;
    unsigned long long passPairs = 0, passTests = 0, passRows = 0, passPartial = 0;
    float passStageMs[STAGE_COUNT] = {};
    long long passValidTris = 0;
    uint32_t *passMasks = nullptr;            // mask buffer for passes when the caller keeps none
    size_t passMasksBytes = 0;
    // triangle ranges of the last frame that needed passes, reused while the
    // same frame (buffers, sizes, bins, light grid, capacity) is launched again
    std::vector<std::pair<long long, long long>> passPlan;
    std::tuple<const void *, const void *, int, int, const void *, const void *, size_t, int, int, long long>
        passKey{};
    // pinned host staging, grown to the largest frame list
    FrameDesc *hFrames = nullptr;
    FrameState *hStates = nullptr;
    int *hBases = nullptr;
    int hCap = 0;
    Counters *hCounters = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t stageEv[STAGE_COUNT + 1] = {};
    // the frame list of the pending / last launch
    std::vector<FrameSpec> frames;
    int maxS = 0, maxT = 0, maxV = 0;
    int launches = 0;
    bool pending = false;
    int replans = 0;
    float lastMs = 0.f;
    // graph of the last launch shape
    cudaGraphExec_t graph = nullptr;
    GraphKey graphKey{};
    bool lastFromGraph = false;
    long long graphCaptures = 0, graphReplays = 0;
    // Look-back tags: launches since the status words were last cleared (the
    // device epoch word, advanced by k_init, holds the same count).  The words
    // are cleared when the arena is laid out anew (they may then hold other
    // buffers' bytes) and before the count reaches kEpochLimit, so a tag never
    // wraps round to the tag of a stale word.
    uint32_t epochCount = 0;
    std::tuple<const void *, size_t, const void *, int, const void *> statusLayout{};
    // Open-box cull (FDZB_OPEN_BOX_*): in auto mode the first launch of a
    // launch shape (frames, samples, triangles, bins) runs the cull's kernel
    // and counts the staged pairs it skips; the shape keeps the cull only if
    // it skipped at least kOpenBoxKeep of them.  Decisions are kept per shape
    // (an engine that alternates between shapes probes each once).
    using BoxShape = std::tuple<int, long long, long long, long long>;
    int openBoxMode = FDZB_OPEN_BOX_AUTO;
    std::map<BoxShape, bool> openBoxKeep;
    BoxShape lastShape{-1, 0, 0, 0};
    bool lastOpenBox = false;
};

constexpr double kOpenBoxKeep = 0.25;

// Launches between two clearings of the look-back words: the sort tags are
// epoch * 16 + (4 x sort slot + pass) in 32 bits, so the epoch stays below 2^28.
constexpr uint32_t kEpochLimit = FDZB_LOOKBACK_EPOCH_LIMIT;

int engine_init(Engine &e, int device);
void engine_release(Engine &e);
// Enqueues e.frames (checked) without waiting.
int engine_enqueue(Engine &e);
// Launch entry of contexts and batches: a single frame known to need triangle
// passes runs them at once (synchronously); anything else is engine_enqueue.
int engine_launch(Engine &e);
// Waits for the pending launch; re-runs it if the pair buffer overflowed.
int engine_sync(Engine &e);
// Statistics of frame i of the last completed launch / of the whole launch.
void frame_stats(const Engine &e, int i, fdzb_frame_stats &o);
void launch_stats(const Engine &e, fdzb_frame_stats &o);
// Device arena bytes a launch of `frames` needs with the given pair capacity.
size_t launch_bytes(const std::vector<FrameSpec> &frames, long long pairCapacity, bool debug);
// Pair capacity an engine starts from for T triangles (grown on overflow).
long long default_pair_capacity(long long T);
// Frame descriptor of the public API to a FrameSpec (light setup on the host).
int desc_to_spec(const fdzb_frame_desc &d, FrameSpec &f, int i);
// Bin grid before any tuning: about 128 samples per bin.
int heuristic_bins(long long S);
void drop_graph(Engine &e);
// Waits for the engine's stream and frees its arena (the next launch allocates anew).
void engine_free_arena(Engine &e);

// Autotuner table: for a size class (ceil(log2 samples), ceil(log2 triangles),
// light grid), the bins per side and the occlusion shape (staged triangles per
// chunk, samples per warp item).
using TuneKey = std::tuple<int, int, int>;
struct TuneChoice {
    int bins = 0;
    int chunk = 32;
    int item = 32;
};
using TuneTable = std::map<TuneKey, TuneChoice>;
TuneKey tune_key(long long S, long long T, int N);
// The tuned choice of f's class, else the heuristic grid and the default shape.
TuneChoice tuned_shape(const TuneTable &table, const FrameSpec &f);
// Tunes every class of `frames` missing from `table` (runs launches on e).
int autotune_bins(Engine &e, TuneTable &table, const std::vector<FrameSpec> &frames, float *scratch,
                  size_t scratchFloats, long long *launches);
// True for a supported occlusion shape.
bool valid_occ_shape(int chunk, int item);

}  // namespace fdzb
