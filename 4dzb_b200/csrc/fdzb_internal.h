// fdzb_internal.h -- shared host/device definitions of the B200 FDZB pipeline.
//
// One launch processes a batch of frames (a single FD-style frame is a batch of
// one).  Samples, triangles and light-plane bins of all frames are laid out back
// to back in HBM, so the binning, sorting and occlusion stages run over one
// global index space: global bin = frame.binBase + local bin, and the unbinned
// key is the total bin count.
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

namespace fdzb {

constexpr float kF32Max = 3.402823466e+38f;   // FD_F32_MAX, FS/util/Util.h:59
constexpr int kMaxLightN = 64;                 // light grid rows / columns (64-bit row words)
constexpr int kMaxLightN32 = 32;               // U32 row words (K/Step5_2_shadowCalPerSample.inl:251)
constexpr int kMaxBins = 512;                  // bins per side

// Light block derived on the host (FS/api.cpp:303-400), device copy per frame.
struct LightParams {
    float mat[16];          // column-major upRight-corner projection
    float RF[2];            // RectangleFactor
    float ur[3], ul[3], dl[3], dr[3];  // light corners
    float xd[3], yd[3];     // x_delt, y_delt
    // A sample's mask has N rows (light samples along x_delt, lightResWidth of
    // them) of NC bits (along y_delt, lightResHeight); bit r * NC + c.  For the
    // reference's square grids N == NC.
    int N;                  // rows (lightResWidth)
    int NC;                 // columns (lightResHeight)
    uint32_t full;          // NC low bits set, when NC <= 32
    unsigned long long fullRows, fullCols;  // N and NC low bits set
};

// Per-frame inputs, outputs and batch offsets (host-filled).
struct FrameDesc {
    const float4 *pos;
    const float4 *nrm;
    const float *vtx;
    const int32_t *idx;
    float *shadow;
    uint32_t *masks;        // nullable
    int W, H, log2up;       // view; log2up = ceil(log2 W) (FS/api.cpp:209)
    int V, vstride, T;      // vertices, floats per vertex, triangles
    int Wb, log2Wb, numBins;
    int cull;
    float esp;
    int maskWords;
    int sampleBase, triBase, binBase;
    int accumulate;         // 1: OR into the masks already in `masks` (later triangle passes)
    LightParams light;
    int hasXform;           // 1: vertices are read through `xform`
    float xform[16];        // column-major model transform (K/moveModel.inl:4-12), applied on read
    // occlusion shape of the frame: triangles staged per chunk (8, 16 or 32)
    // and samples per warp work item (32, 64 or 128: a warp takes the item's
    // samples 32 at a time, so larger items mean fewer warps per bin)
    int occChunk, occItem;
};

// Slots of FrameState::acc (order-preserving uint32 encodings of floats).
enum AccSlot {
    ACC_SMAXW = 0,   // max light depth over non-background samples (k1)
    ACC_TMAXW,       // max light depth over all vertices (k2)
    ACC_S_MINU, ACC_S_MINV, ACC_S_MINW, ACC_S_MAXA, ACC_S_MAXB, ACC_S_MAXW,  // front samples (k3)
    ACC_M_MINU, ACC_M_MINV, ACC_M_MINW, ACC_M_MAXA, ACC_M_MAXB, ACC_M_MAXW,  // vertices (k4)
    ACC_COUNT
};

// Per-frame values computed on the device.
struct FrameState {
    uint32_t acc[ACC_COUNT];
    int nFront;             // non-background front-facing samples
    int state;              // 0 / 1 / 2 (see fdzb_frame_stats)
    int nValidTris;
    int nValidSamples;
    float f, subx, suby;
    float Bx, By, Bz, Ex, Ey, Ez;
    float fx, fy;
    float sampleAabb[6], modelAabb[6];
    int quirkKeyRange;
    int pad[3];
};

// Launch-wide counters and error word (zeroed every launch).
struct Counters {
    int pairCount;          // triangle/bin pairs produced
    int pairOverflow;       // 1 if pairCount > capacity
    int itemCount;          // occlusion work items
    int itemCursor;         // occlusion work queue head
    int triTileCounter;     // look-back scan tile ticket
    int errorFlags;         // bit 0: look-back wait gave up, bit 1: mbarrier wait gave up
    unsigned long long pairTests;
    int sortTileCounter[12]; // one ticket per radix pass (4 sample, 4 pair, 4 triangle)
    unsigned long long rowsEvaluated;   // light rows evaluated by pair tests
    unsigned long long partialMasks;    // row masks that needed the ceil(-D/B) threshold
    unsigned long long pairsExamined;   // sample/triangle pairs reaching the AABB pre-cull (the
                                        // open-box kernel: staged triangles its lanes take up)
    unsigned long long chunks;          // staged triangle chunks (warp-level)
    unsigned long long rounds;          // compute rounds of 32 pair slots (k_occlusion_pairs)
    unsigned long long boxSkips;        // pairs the open-box cull skipped (warp union or the lane's box)
};

// Stage boundaries recorded when per-stage timing is on.
enum StageId { STAGE_SETUP = 0, STAGE_SAMPLE_SORT, STAGE_TRI_PAIRS, STAGE_PAIR_SORT, STAGE_OCCLUSION,
               STAGE_COUNT };

// Start of a segment no element reached (the bins' sample and triangle
// segments are built by atomic minima and maxima from this value and 0).
constexpr int kSegAbsent = 0x7FFFFFFF;

enum ErrorBits { ERR_LOOKBACK_TIMEOUT = 1, ERR_MBAR_TIMEOUT = 2, ERR_BAD_INPUT = 4, ERR_INTERNAL = 8 };

// Device buffers of one launch (carved from one arena).
struct DeviceBuffers {
    FrameDesc *frames;        // [nframes]
    FrameState *states;       // [nframes]
    Counters *counters;
    int nframes;
    int totalSamples, totalTris, totalBins;
    int pairCapacity;
    // samples
    uint32_t *keysA, *valsA, *keysB, *valsB;   // [totalSamples]
    int32_t *binSampleStart, *binSampleEnd;    // [totalBins + 1]
    uint32_t *binStat;                          // [8 * totalBins] ordered encodings: maxz, Rx, Ry, Rz, Rw, 3 pad
    // triangles
    float4 *triRec;                             // [4 * totalTris]
    float4 *triPrj;                             // [2 * totalTris] vertex projections (open-box test)
    int32_t *triCount;                          // [totalTris]
    unsigned long long *triScanStatus;          // [triTiles] epoch-tagged look-back words
    // pairs
    uint32_t *pkeysA, *pvalsA, *pkeysB, *pvalsB;  // [pairCapacity]
    int32_t *binTriStart, *binTriEnd;          // [totalBins]
    // coverage order: (bucket, triangle) pairs sorted by bucket; the sorted
    // values are the order in which k_tri_pairs emits the triangles' pairs
    uint32_t *tkeysA, *tvalsA, *tkeysB, *tvalsB;  // [totalTris]
    // sort scratch
    uint32_t *sortHist;                         // [12 * 256]: 4 sample, 4 pair, 4 triangle passes
    unsigned long long *sortStatus;             // [sortStatusTiles * 256] epoch-tagged
    size_t sortStatusTiles;
    int *sampleBases, *triBases, *binBases;     // [nframes] ascending global bases
    // occlusion work list
    int4 *items;                                // [itemCapacity]
    int itemCapacity;
    // sorted data lands in the A buffers after an even number of passes, B after odd
    int samplePasses, pairPasses, triPasses;
    int pairTriBits;                            // > 0: pairs are words bin << pairTriBits | triangle
    int depthBits;                              // coverage-bucket bits of the triangle order (0:
                                                // the reference's order, no triangle sort)
    int occVariant;                             // 0: k_occlusion (lane per sample), 1: k_occlusion_pairs
    int rayCast;                                // 1: ray-cast cross-check (REF_CAL) instead of edge masks
    int wide;                                   // 1: some frame's light grid exceeds 32 rows or
                                                // columns: 64-bit row words
    int depthPlane;                             // 1: the frames test each triangle's own plane
    int openBox;                                // 1: the occlusion kernel with the open-box cull
    int countWork;                              // 1: the occlusion kernel that accumulates the work counters
    int rows16;                                 // 1: every grid of the launch has at most 16 rows
    uint32_t *epochWord;                        // launch sequence number (look-back tags), advanced
                                                // on the device by k_init so graph replays stay fresh
    // debug capture (nullptr unless enabled): pre-sort copies of the key/value arrays
    uint32_t *dbgKeys, *dbgVals, *dbgPKeys, *dbgPVals;
};

// Host side.
void light_setup(const float rightRadius, const float topRadius, const float position[3],
                 const float viewDir[3], const float upDir[3], int resW, int resH,
                 LightParams *out);

// Kernel drivers (fdzb_pipeline.cu).  All enqueue on `stream`, no host syncs.
// maxS / maxT / maxV: largest per-frame sample / triangle / vertex counts.
// stageEvents: nullptr, or STAGE_COUNT + 1 events recorded at the stage
// boundaries.  *launches receives the number of kernels enqueued.
cudaError_t run_pipeline(const DeviceBuffers &b, int maxS, int maxT, int maxV, cudaStream_t stream,
                         cudaEvent_t *stageEvents, int *launches);
// Issue-rate probe: lane FP32 adds per second of a kernel with independent chains.
cudaError_t measure_alu_rate(double *laneOpsPerSecond);
cudaError_t check_division(unsigned long long trials, unsigned long long seed, unsigned long long *mismatches,
                           unsigned long long *checked);

// Records `msg` as this thread's fdzb_last_error() and returns `code`.
int set_error(int code, const std::string &msg);
int sort_passes_for(long long keyRangeExclusive);
cudaError_t run_move_model(float *vtx, int vstride, int V, const float m[16], cudaStream_t stream);
#ifndef FDZB_SORT_ITEMS
#define FDZB_SORT_ITEMS 16
#endif
constexpr int kSortTileHost = 256 * FDZB_SORT_ITEMS;   // keys per radix-sort tile (fdzb_sort.cuh)
constexpr int kTriTileHost = 64;      // triangles per pair-scan tile (the smaller of the two sizes)
constexpr int kSortSlots = 3;        // radix sorts per launch: samples, pairs, triangles

}  // namespace fdzb
