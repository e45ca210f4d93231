/*
 * fdzb.h -- C ABI of the B200 FDZB soft-shadow library (libfdzb.so).
 *
 * Drop-in boundary for the FD:: entry points of 4DZB's soft-shadow core
 * (4DZB/FDZB_Soft_Shadow/api.h:10-56).  Each global-context function below keeps
 * the shape of the reference function named beside it; GL object handles are
 * replaced by caller-owned device pointers (the reference maps its GL VBO/IBO,
 * G-buffer textures and PBO into exactly such pointers every frame,
 * FS/api.cpp:413-420 and FS/util/OpenGLinteroperate.h:42-55,131-136).
 *
 * Conventions
 *  - every entry point returns int status: 0 = FDZB_OK, negative = error;
 *    fdzb_last_error() returns the message of the last failure on this thread;
 *  - no C++ exceptions cross the ABI; no torch types appear in any signature;
 *  - device pointers are CUDA global-memory pointers on the context's device;
 *  - samples are row-major float4[W*H] positions and normals (xyz, w unused),
 *    NaN position.x marks background (the reference's G-buffer clear value);
 *  - outputs: shadow float[W*H] at index y*W+x (fraction of occluded light
 *    samples, 1 - visibility) and, optionally, masks uint32[W*H][ceil(Lw*Lh/32)]
 *    for an Lw x Lh light grid, with light sample (row i < Lw along the
 *    light's width, column j < Lh along its height) at bit i*Lh+j, least
 *    significant bit first (square grids: bit i*N+j).
 *
 * Reference-shaped global context: one process-wide context on the current CUDA
 * device, single-threaded like FD:: (K/FourD.cu:47-136).  The fdzb_ctx_* handle
 * API is the re-entrant form: one context per scene / host thread / stream.
 */
#ifndef FDZB_H
#define FDZB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDZB_OK                   0
#define FDZB_ERR_INVALID_ARG     -1
#define FDZB_ERR_CUDA            -2
#define FDZB_ERR_NOT_INITIALIZED -3
#define FDZB_ERR_NO_MEMORY       -4
#define FDZB_ERR_CAPACITY        -5   /* a device buffer overflowed and re-planning failed */
#define FDZB_ERR_DEVICE_TIMEOUT  -6   /* a bounded device-side wait gave up */
#define FDZB_ERR_UNSUPPORTED     -7
#define FDZB_ERR_NOT_READY       -8   /* required inputs (view, samples, model, light, output) not set */

/* Same 52-byte layout as AreaLightDes (4DZB/FDZB_Soft_Shadow/AreaLightDesc.h:3-14):
 * two floats, three glm::vec3, two ints.  The reference runs square grids,
 * lightResWidth == lightResHeight = N in 1..32; this library takes any
 * lightResWidth x lightResHeight in 1..64 each.  A sample's mask has
 * lightResWidth rows (light samples along x_delt) of lightResHeight bits (along
 * y_delt): bit r * lightResHeight + c, LSB first, ceil(W*H/32) words. */
typedef struct fdzb_area_light_desc {
    float rightRadius;      /* half width */
    float topRadius;        /* half height */
    float position[3];
    float viewDir[3];
    float upDir[3];
    int32_t lightResWidth;
    int32_t lightResHeight;
} fdzb_area_light_desc;

/* ---- reference-shaped global context (FD:: namespace, FS/api.h) ---------- */

/* FD::FDinit (FS/api.h:15, FS/api.cpp:48-144). Creates the global context on the
 * current device.  Calling it again resets the context. */
int fdzb_init(void);
/* FD::FDsetBackfaceCull (FS/api.h:18, FS/api.cpp:146-150).  Default 1, like
 * m_enable_backfacecull (K/FourD.cu:61). */
int fdzb_set_backface_cull(int enable);
/* FD::FDaddModel (FS/api.h:21, FS/api.cpp:152-160).  d_vtx: n_vtx vertices of
 * vtx_stride_bytes each (xyz first; stride a multiple of 4 bytes), d_idx: int3[n_tri].
 * Like the reference (FS/api.cpp:430-445) only the first model added is shaded. */
int fdzb_add_model(const float *d_vtx, size_t n_vtx, size_t vtx_stride_bytes,
                   const int32_t *d_idx, size_t n_tri, const char *name);
/* FD::FDsetSampleGLTex (FS/api.h:24, FS/api.cpp:162-166): the G-buffer position and
 * normal images, as device float4[W*H] arrays. */
int fdzb_set_sample_buffers(const float *d_pos, const float *d_nrm);
/* FD::FDsetOutputGLBuffer (FS/api.h:27, FS/api.cpp:168-171): float[W*H] shadow
 * fractions; d_masks (nullable) receives the per-sample occlusion bit masks. */
int fdzb_set_output_buffer(float *d_shadow, uint32_t *d_masks);
/* FD::FDregisterGLres / FDunregisterGLres (FS/api.h:30-33, FS/api.cpp:173-191).  No
 * graphics interop here: these validate that the buffers set above are
 * device-accessible and return 0. */
int fdzb_register_resources(void);
int fdzb_unregister_resources(void);
/* FD::FDsetBinNum (FS/api.h:36; body commented out at FS/api.cpp:193-202, the
 * reference fixes 16 at compile time, FS/constants.h:13).  Light-plane bins per
 * side; power of two in [1, 512].  Default 16. */
int fdzb_set_bin_num(size_t bin_num);
/* FD::FDsetView (FS/api.h:39, FS/api.cpp:205-237). */
int fdzb_set_view(int view_width, int view_height);
/* FD::FDsetScenesEsp (FS/api.h:41, FS/api.cpp:238-241).  Default 1e-6 like
 * K/FourD.cu:62 (the demo app sets 1e-3). */
int fdzb_set_scenes_esp(float scenes_esp);
/* FD::FDsetSceneParams (FS/api.h:44, FS/api.cpp:243-294): capacity hints used to
 * pre-size per-triangle buffers. */
int fdzb_set_scene_params(size_t max_triangle_num, size_t max_vertices_num);
/* FD::FDsetAreaLight (FS/api.h:49, FS/api.cpp:303-400). */
int fdzb_set_area_light(const fdzb_area_light_desc *light);
/* FD::FDLaunch (FS/api.h:52, FS/api.cpp:402-582): computes one frame and returns its
 * GPU time in milliseconds (CUDA events around the whole frame), or a negative
 * FDZB_ERR_* value on failure. */
float fdzb_launch(void);
/* FD::moveModel (FS/api.h:12, K/moveModel.inl:31-51): applies the column-major
 * 4x4 matrix m to the xyz of every vertex of model 0, in place. */
int fdzb_move_model(const float m[16]);
/* Message of the last failing call on this thread ("" if none). */
const char *fdzb_last_error(void);

/* ---- context handle API (re-entrant form) -------------------------------- */

typedef struct fdzb_ctx fdzb_ctx;

/* Per-frame counters of the last completed launch. */
typedef struct fdzb_frame_stats {
    int32_t state;             /* 0: no sample or vertex in front of the light;
                                  1: only back-facing samples shaded (no light plane,
                                     no valid sample or triangle); 2: full pipeline */
    int32_t valid_samples;     /* samples with a light-plane bin */
    int32_t valid_triangles;   /* triangles overlapping the light plane */
    int32_t num_pairs;         /* triangle/bin pairs */
    int32_t num_bins;
    int32_t pair_capacity;
    int64_t pair_tests;        /* sample/triangle pairs past the AABB pre-cull (counted with
                                  profiling on, fdzb_ctx_set_profiling; 0 otherwise) */
    float f;                   /* far plane */
    float sub[2];
    float lp_begin[3], lp_end[3], lp_factor[2];
    float sample_aabb[6], model_aabb[6];
    int32_t replans;           /* pair-buffer regrowths in this launch */
    int32_t quirk_key_range;   /* samples whose bin fell outside the grid (treated as unbinned) */
    int32_t kernel_launches;   /* kernels enqueued by the frame */
    int32_t triangle_passes;   /* 1, or the passes over triangle ranges of a frame whose pairs
                                  exceeded the pair-capacity limit */
    int64_t rows_evaluated;    /* light-grid rows evaluated by pair tests (profiling on) */
    int64_t partial_masks;     /* row masks that needed the ceil(-D/B) threshold (profiling on) */
    float stage_ms[5];         /* with profiling on: setup, sample sort, triangle pairs,
                                  pair sort, occlusion+shading (CUDA events) */
    float pad1;
} fdzb_frame_stats;

/* device < 0: current device. */
int fdzb_ctx_create(fdzb_ctx **out, int device);
int fdzb_ctx_destroy(fdzb_ctx *ctx);
/* Work is enqueued on `stream` (a cudaStream_t); NULL = the context's own stream. */
int fdzb_ctx_set_stream(fdzb_ctx *ctx, void *stream);
int fdzb_ctx_set_backface_cull(fdzb_ctx *ctx, int enable);
int fdzb_ctx_add_model(fdzb_ctx *ctx, const float *d_vtx, size_t n_vtx, size_t vtx_stride_bytes,
                       const int32_t *d_idx, size_t n_tri, const char *name);
int fdzb_ctx_set_sample_buffers(fdzb_ctx *ctx, const float *d_pos, const float *d_nrm);
int fdzb_ctx_set_output_buffer(fdzb_ctx *ctx, float *d_shadow, uint32_t *d_masks);
int fdzb_ctx_set_bin_num(fdzb_ctx *ctx, size_t bin_num);
int fdzb_ctx_set_view(fdzb_ctx *ctx, int view_width, int view_height);
int fdzb_ctx_set_scenes_esp(fdzb_ctx *ctx, float scenes_esp);
int fdzb_ctx_set_scene_params(fdzb_ctx *ctx, size_t max_triangle_num, size_t max_vertices_num);
int fdzb_ctx_set_area_light(fdzb_ctx *ctx, const fdzb_area_light_desc *light);
int fdzb_ctx_move_model(fdzb_ctx *ctx, const float m[16]);
/* Shadow method (the reference chooses at compile time, REF_CAL in
 * K/FourD.h:17, FS/api.cpp:545-552).
 *   FDZB_SHADOW_EDGE_MASKS (default): the 4D-Z-buffer edge-function row masks
 *     (K/Step5_2_shadowCalPerSample.inl);
 *   FDZB_SHADOW_RAY_CAST: the reference's ray-cast cross-check (refCal_kernel,
 *     K/Step5_2_calRef.inl): one ray per light sample through each triangle of
 *     the sample's bin.  Same bins and lists; masks in this library's layout
 *     (the reference numbers light samples transposed).  Much slower; meant to
 *     cross-check the edge-function result, which it matches except for light
 *     samples on or next to a projected triangle edge. */
#define FDZB_SHADOW_EDGE_MASKS 0
#define FDZB_SHADOW_RAY_CAST   1
int fdzb_ctx_set_shadow_method(fdzb_ctx *ctx, int method);

/* Depth plane (edge-function masks only; default off).  The reference's
 * per-sample kernel assumes every occluder lies between the sample and the
 * light (it has no triangle-plane test), and shadows wrongly with occluders
 * beside or behind the light.  Enabled, a pair whose triangle reaches the
 * light plane (min light depth <= 0) or the sample's depth also tests the
 * triangle's own plane, as the reference's per-bin kernel does
 * (K/Step5_2_shadowCal.inl:667-674, 838): light samples on the sample's side
 * of that plane are not occluded by it. */
int fdzb_ctx_set_depth_plane(fdzb_ctx *ctx, int enable);

/* Model transform applied to model 0's vertices as they are read, leaving the
 * vertex buffer untouched (the reference's moveModel rewrites the VBO in place,
 * K/moveModel.inl:14-50).  m: column-major 4x4, NULL = none.  A launch with m
 * gives bit for bit what fdzb_ctx_move_model(ctx, m) followed by a launch
 * gives on the untransformed buffer; unlike moveModel it does not accumulate,
 * so an animated scene passes each frame's full transform.  No host sync. */
int fdzb_ctx_set_model_transform(fdzb_ctx *ctx, const float m[16]);
/* Synchronous frame (FDLaunch form); *ms_out (nullable) gets the GPU time. */
int fdzb_ctx_launch(fdzb_ctx *ctx, float *ms_out);
/* Enqueue the frame on the context stream without waiting.  Pair-buffer overflow
 * is only detected (and the frame re-run) by fdzb_ctx_sync. */
int fdzb_ctx_launch_async(fdzb_ctx *ctx);
int fdzb_ctx_sync(fdzb_ctx *ctx);
int fdzb_ctx_get_stats(fdzb_ctx *ctx, fdzb_frame_stats *out);

/* Intermediate arrays of the last launch, for parity checks and debugging (the
 * reference dumps the same data with saveBinImage / showBinTriPair,
 * K/binRaster.inl:61-182, K/Step4_RasterizeTriangleToBin.inl:236-250).
 * Copies `bytes` bytes of array `what` into host memory `dst`. */
enum fdzb_array_id {
    FDZB_ARR_SAMPLE_KEYS = 0,       /* int32[S] bin key per sample, y*W+x order (num_bins = unbinned) */
    FDZB_ARR_SORTED_SAMPLE_KEYS,    /* int32[S] */
    FDZB_ARR_SORTED_SAMPLE_IDS,     /* int32[S] y*W+x of each sorted entry */
    FDZB_ARR_BIN_SAMPLE_START,      /* int32[num_bins+1] */
    FDZB_ARR_BIN_SAMPLE_END,        /* int32[num_bins+1] */
    FDZB_ARR_BIN_MAXZ,              /* float[num_bins] */
    FDZB_ARR_BIN_RANGE,             /* float[4*num_bins] */
    FDZB_ARR_TRI_COUNT,             /* int32[T] bins per triangle */
    FDZB_ARR_PAIR_BIN,              /* int32[num_pairs] triangle order */
    FDZB_ARR_PAIR_TRI,              /* int32[num_pairs] */
    FDZB_ARR_SORTED_PAIR_BIN,       /* int32[num_pairs] */
    FDZB_ARR_SORTED_PAIR_TRI,       /* int32[num_pairs] */
    FDZB_ARR_BIN_TRI_START,         /* int32[num_bins] */
    FDZB_ARR_BIN_TRI_END,           /* int32[num_bins] */
    FDZB_ARR_TRI_AABB,              /* float[8*T] (min xyz,1, max xyz,1) */
    FDZB_ARR_WORK_COUNTERS,         /* uint64[7] occlusion work: pair tests, light rows, partial row
                                       masks (these three with profiling on), pairs reaching the
                                       AABB pre-cull, triangle chunks,
                                       compute rounds (these three: counted by the pair-compacting
                                       occlusion kernel only), pairs skipped by the open-box cull */
    FDZB_ARR_COUNT
};
int fdzb_ctx_export(fdzb_ctx *ctx, int what, void *dst, size_t bytes);
/* flags bit 0: keep copies of the pre-sort key/value arrays (FDZB_ARR_SAMPLE_KEYS,
 * FDZB_ARR_PAIR_BIN, FDZB_ARR_PAIR_TRI) at the cost of two extra device copies per
 * sort.  Bit 1: keep triangle/bin pairs as separate key and value arrays even
 * where one 32-bit word (bin << b | triangle) would hold a pair -- the packed
 * form sorts keys alone; both give the same lists (this switch exists to test
 * both).  Off by default. */
int fdzb_ctx_set_debug(fdzb_ctx *ctx, int flags);

/* Order of each bin's triangle list (no counterpart in the reference, whose
 * thrust::sort_by_key leaves ascending triangle ids inside a bin,
 * K/Step4_RasterizeTriangleToBin.inl:220-223).  Masks and shadows are identical in
 * both orders -- a sample's mask is the OR over its bin's triangles -- only the
 * number of pair tests before a sample's light is fully blocked changes.
 *   FDZB_TRI_ORDER_REFERENCE: the reference's order (parity of the sorted lists);
 *   FDZB_TRI_ORDER_COVERAGE (default): largest angular size first (triangle area
 *     over the squared light-depth distance from the far plane to its top vertex). */
#define FDZB_TRI_ORDER_REFERENCE 0
#define FDZB_TRI_ORDER_COVERAGE  1
#define FDZB_TRI_ORDER_DEPTH     FDZB_TRI_ORDER_COVERAGE   /* earlier name of the same value */
int fdzb_ctx_set_tri_order(fdzb_ctx *ctx, int order);

/* Warp schedule of the occlusion stage (no counterpart in the reference, which
 * runs one thread per sample, K/Step5_2_shadowCalPerSample.inl:37-231).  Results
 * are identical; only the speed differs.
 *   FDZB_OCC_LANE_PER_SAMPLE (default): a lane per sample of a bin, the warp
 *     streaming the bin's triangles through shared memory;
 *   FDZB_OCC_LANE_PER_PAIR: the pairs that pass the AABB pre-cull, and then
 *     their (pair, light row) units, are dealt one per lane.  Square grids up
 *     to 32 x 32 without the depth plane; other launches run lane per sample. */
#define FDZB_OCC_LANE_PER_SAMPLE 0
#define FDZB_OCC_LANE_PER_PAIR   1
int fdzb_ctx_set_occlusion_schedule(fdzb_ctx *ctx, int schedule);

/* Largest triangle/bin pair buffer (pairs; default and maximum 2^29, 8 GB of
 * pair arrays).  No counterpart in the reference, whose fixed 70M-pair buffer
 * overflows unchecked (FS/constants.h:15).  A frame whose pairs exceed it runs
 * in passes over ranges of its triangles whose occlusion bits are OR-ed
 * together (results identical; fdzb_frame_stats.triangle_passes counts them).
 * When the frame has no mask output, the library keeps a mask buffer of its own
 * for the passes. */
int fdzb_ctx_set_pair_capacity_limit(fdzb_ctx *ctx, int64_t pairs);

/* Profiling modes.  FDZB_PROFILE_ALL: per-stage GPU timing (CUDA events
 * between stages, read back in fdzb_frame_stats.stage_ms) and the occlusion
 * kernel's work counters (pair_tests, rows_evaluated, partial_masks: counted
 * only in this mode, by a form of the kernel that accumulates them, a few per
 * cent slower).  FDZB_PROFILE_STAGES: the stage timing alone, with the kernels
 * that run unprofiled.  Off by default; profiled launches are not replayed
 * from a CUDA graph.  The reference times only the whole frame
 * (FS/api.cpp:405-409,574-581). */
#define FDZB_PROFILE_OFF 0
#define FDZB_PROFILE_ALL 1
#define FDZB_PROFILE_STAGES 2
int fdzb_ctx_set_profiling(fdzb_ctx *ctx, int enable);

/* Measures the FP32 issue rate of the current device (lane operations per second
 * of a kernel of independent FP32 add chains): the peak against which the
 * occlusion kernel's operation rate is reported.  No counterpart in the reference. */
int fdzb_measure_alu_rate(double *lane_ops_per_second);

/* Device self-check of the occlusion kernel's row quotient: -D / B from a
 * hoisted reciprocal RN(1/B) by two Markstein correction steps, which the pair
 * test uses in place of the IEEE division where its operands are in range,
 * the reciprocal itself from the hardware approximation and one
 * Newton-Raphson step.  Compares that reciprocal with __frcp_rn for every
 * float of the admitted range (|B| in [2^-100, 2^40), 2.35e9 values), then
 * runs `trials` trials of three cases each (random operands over the admitted
 * ranges, quotients next to rounding midpoints, quotients at small integers)
 * against __fdiv_rn; returns the number of compared values and of results
 * that differ in any bit (expected: 0).  No counterpart in the reference,
 * whose rows divide directly (K/Step5_2_shadowCalPerSample.inl:20). */
int fdzb_check_division(uint64_t trials, uint64_t seed, uint64_t *mismatches, uint64_t *checked);

/* Host-side light setup only (FS/api.cpp:303-400): fills the 16-float
 * column-major light projection, RectangleFactor and the four light corners
 * (upRight, upLeft, downLeft, downRight), x_delt and y_delt. */
int fdzb_light_setup(const fdzb_area_light_desc *light, float mat[16], float rect_factor[2],
                     float corners[12], float deltas[6]);

/* Light-sample positions (host): out[3*(i*W + j) ..] = upRight + x_delt*j +
 * y_delt*i for i < lightResHeight, j < lightResWidth, in the reference's own
 * numbering (FS/api.cpp:351-357, the positions its REF_CAL check and the app's
 * shading use).  out: 3 * W * H floats. */
int fdzb_light_sample_positions(const fdzb_area_light_desc *light, float *out);

/* ---- shading pass --------------------------------------------------------- */

/* Deferred Phong shading of the shadowed frame, the app's consumer of the
 * shadow buffer (4DZB/Resources/shader/phoneShading.shf:25-60): per pixel,
 * the average over the light samples of La*ka + (Ld*kd*max(L.N, 0) +
 * Ls*ks*max(R.V, 0)^shininess) * (1 - shadow), alpha 1.  G-buffer packing as the
 * reference's: g0 = position.xyz | ks.r, g1 = normal.xyz | ks.g, g2 = ka.rgb |
 * ks.b, g3 = kd.rgb | shininess (float4[W*H] each, 16-byte aligned).  Pixels
 * whose shadow is NaN are left untouched (the shader discards them).  FP32 with
 * CUDA's math functions; no bit-exact claim against a GLSL driver.  The app
 * itself shades with one light sample (Render.cpp:461-470, 550). */
typedef struct fdzb_shade_desc {
    int32_t W, H;
    const float *d_g0, *d_g1, *d_g2, *d_g3;
    const float *d_shadow;         /* float[W*H] */
    float *d_rgba;                 /* float4[W*H] */
    float camera_pos[3];
    float La[3], Ld[3], Ls[3];
    int32_t n_light_samples;       /* 1..4096 */
    const float *d_light_samples;  /* device float[3 * n_light_samples] world positions */
} fdzb_shade_desc;
/* Enqueued on `stream` (cudaStream_t, NULL = legacy default); no host sync. */
int fdzb_shade(const fdzb_shade_desc *desc, void *stream);

/* ---- G-buffer rasteriser (the view samples' producer) --------------------- */

/* Replaces the app's GL G-buffer pass (4DZB/Render/Render.cpp:390-431,
 * DrawModel :267-340, shaders 4DZB/Resources/shader/gatherData.shv/.shf) so
 * that real meshes feed fdzb_* without a graphics stack.  One draw rasterises a
 * triangle list (the MeshManager layout, 4DZB/ResourceManager/MeshManager.cpp:
 * 35-89: 8 floats per vertex, position at 0, texcoord at 3, normal at 5) with
 * the depth test GL_LESS; per pixel
 *   g0 = (worldPos, Ks.r)  g1 = (worldN, Ks.g)  g2 = (Ka, Ks.b)  g3 = (Kd, shininess)
 * with worldPos = model * (P, 1), worldN = model * (N, 0) interpolated
 * perspective-correctly, and clip = view_proj * (worldPos, 1) -- the gatherData
 * shaders' outputs, so g0 and g1 are this library's sample position and normal
 * buffers.  Cleared pixels are NaN (the app's clear colour), depth 1.  Rows run
 * bottom to top (row 0 is window y = 0, as in the GL textures the app hands to
 * FDsetSampleGLTex).  The rasterisation rules GL leaves to the implementation
 * are fixed here: near-plane clipping in clip space (far plane and viewport per
 * fragment), window coordinates snapped to 1/16 pixel, coverage at pixel
 * centres with exact 64-bit edge functions and a rule that gives a centre on a
 * shared edge to exactly one triangle, both windings drawn, ties in depth won
 * by the earlier triangle.  Textured materials (the shader's NaN colour ->
 * texture lookup) are not supported: materials are constant colours.
 * Sub-triangles with a vertex beyond 2^26 pixels of the viewport are dropped
 * and counted. */
typedef struct fdzb_raster fdzb_raster;
typedef struct fdzb_raster_desc {
    const float *d_vtx;            /* n_vtx vertices, vtx_stride_bytes apart */
    int32_t n_vtx;
    int32_t vtx_stride_bytes;      /* multiple of 4; 32 for the MeshManager layout */
    int32_t pos_offset, nrm_offset;/* in floats: 0 and 5 for the MeshManager layout */
    const uint32_t *d_idx;         /* 3 per triangle */
    int32_t n_tri;
    const int32_t *d_tri_material; /* nullable: every triangle uses material 0 */
    const float *d_materials;      /* n_materials x 10 floats: Ka rgb, Kd rgb, Ks rgb, shininess */
    int32_t n_materials;
    float model[16];               /* column-major modelMatrix */
    float view_proj[16];           /* column-major ViewAndPerspectiveMatrix */
    int32_t W, H;                  /* 1..16384 */
    int32_t clear;                 /* 1: clear the G-buffer (NaN) and depth (1) first; 0: draw on
                                      top of an earlier draw (needs the same d_depth) */
    float *d_g0, *d_g1;            /* float4[W*H], 16-byte aligned */
    float *d_g2, *d_g3;            /* nullable float4[W*H] */
    float *d_depth;                /* float[W*H] window depth; nullable only with clear */
} fdzb_raster_desc;
typedef struct fdzb_raster_stats {
    int64_t triangles, sub_triangles, dropped, tile_pairs, bad_indices, bad_materials;
    int32_t tiles_x, tiles_y;
    float ms;                      /* last draw, device time */
    float pad;
} fdzb_raster_stats;
int fdzb_raster_create(fdzb_raster **out, int device);
int fdzb_raster_destroy(fdzb_raster *r);
/* stream: a cudaStream_t; NULL = the rasteriser's own stream. */
int fdzb_raster_set_stream(fdzb_raster *r, void *stream);
/* Enqueues one draw.  Waits once on the stream for the tile-list size, then
 * returns with the rasterisation in flight; fdzb_raster_sync waits for it. */
int fdzb_raster_draw(fdzb_raster *r, const fdzb_raster_desc *desc);
int fdzb_raster_sync(fdzb_raster *r);
int fdzb_raster_get_stats(fdzb_raster *r, fdzb_raster_stats *stats);

/* Library version string. */
const char *fdzb_version(void);

/* CUDA graphs (no counterpart in the reference, which issues each kernel, sort
 * and read-back of FDLaunch separately, FS/api.cpp:405-575).  On by default: a
 * launch is captured once per launch shape (frame count, sizes, bin totals,
 * pair capacity, stream) and replayed while the shape is unchanged.  Graphs
 * are not used with profiling or debug capture on, or on the legacy default
 * stream. */
int fdzb_ctx_set_graph(fdzb_ctx *ctx, int enable);

/* Occlusion shape, no counterpart in the reference (its per-sample kernel runs
 * one thread per sample, K/Step5_2_shadowCalPerSample.inl:236-260): chunk =
 * triangles of a bin's list staged in shared memory per round (8, 16 or 32,
 * default 32); item = samples of one bin per warp work item (32, 64 or 128,
 * default 32; a warp takes an item's samples 32 at a time, so larger items
 * put fewer warps on a bin).  Results are identical for every shape; the
 * batch and server autotuners pick it per size class. */
int fdzb_ctx_set_occlusion_shape(fdzb_ctx *ctx, int chunk, int item);

/* Open-box cull, no counterpart in the reference: once some of a sample's
 * light rows or columns are full, a pair whose triangle cannot reach the box
 * of its still-unset light samples (a test on the triangle's projected
 * vertices, with a margin far above FP32 rounding) is skipped; masks and
 * shadows are identical (the mask is the OR over the bin's triangles).  It
 * runs in its own instantiation of the occlusion kernel, which is faster where
 * samples end in umbra and slower where they stay in penumbra.  AUTO (the
 * default): the first launch of each launch shape (frames, samples, triangles,
 * bins) runs it and counts the staged pairs it skips; the shape keeps it only
 * if that is at least a quarter of them.  Edge-function masks only. */
#define FDZB_OPEN_BOX_OFF 0
#define FDZB_OPEN_BOX_ON 1
#define FDZB_OPEN_BOX_AUTO 2
int fdzb_ctx_set_open_box(fdzb_ctx *ctx, int mode);

/* Testing aids, no counterpart in the reference.  The sorts' decoupled
 * look-back tags its status words with the context's launch number (a device
 * word advanced by every launch; FS/api.cpp:402-582 has no look-back: Thrust's
 * sorts run there).  The words are never cleared between launches, except
 * when the arena is laid out anew and before the launch number reaches
 * FDZB_LOOKBACK_EPOCH_LIMIT, when they and the number restart from zero, so a
 * tag never wraps round to a stale word's.  set_launch_epoch moves the number
 * (after a first launch; value < the limit) so that tests can cross that
 * point; get_launch_epoch reads it after the pending launch. */
#define FDZB_LOOKBACK_EPOCH_LIMIT 0x0FFFFFFFu
int fdzb_ctx_set_launch_epoch(fdzb_ctx *ctx, uint32_t value);
int fdzb_ctx_get_launch_epoch(fdzb_ctx *ctx, uint32_t *out);

/* ---- batches: many independent frames per launch ------------------------- */

/* No counterpart in the reference, which renders one frame per FD::FDLaunch
 * (FS/api.cpp:405-575).  A batch runs a list of independent frames -- each with
 * its own view samples, triangle soup, light and bin grid -- through one launch
 * per pipeline stage: the frames' samples, triangles and bins are laid end to
 * end in HBM and every stage processes all of them at once.  Each frame's
 * results are identical to a separate fdzb_ctx_launch of the same inputs. */
typedef struct fdzb_frame_desc {
    const float *d_pos;            /* float4[W*H] row-major, NaN x = background */
    const float *d_nrm;            /* float4[W*H] */
    int32_t W, H;
    const float *d_vtx;            /* vertices: xyz at the start of every stride */
    size_t n_vtx;
    size_t vtx_stride_bytes;
    const int32_t *d_idx;          /* int3 per triangle */
    size_t n_tri;
    fdzb_area_light_desc light;    /* width x height grid, each in [1, 64] */
    int32_t bins;                  /* bins per side: power of two in [1, 512]; 0 = autotuned */
    int32_t cull;                  /* back-face culling of triangles (FDsetBackfaceCull) */
    float esp;                     /* FDsetScenesEsp */
    float *d_shadow;               /* float[W*H] at y*W+x */
    uint32_t *d_masks;             /* nullable: uint32[W*H*ceil(Lw*Lh/32)], bit r*Lh+c */
    const float *model_transform;  /* nullable host pointer: 16 floats, see fdzb_ctx_set_model_transform */
} fdzb_frame_desc;

typedef struct fdzb_batch fdzb_batch;

typedef struct fdzb_batch_stats {
    fdzb_frame_stats totals;       /* launch-wide: sums over frames (state = 2) */
    int32_t frames;
    int32_t from_graph;            /* last launch replayed or captured a graph */
    int64_t graph_captures;
    int64_t graph_replays;
    int32_t tuned_classes;         /* size classes with an autotuned bin grid */
    int32_t pad0;
    int64_t tune_launches;
    float ms;                      /* GPU time of the last launch */
    float pad1;
} fdzb_batch_stats;

int fdzb_batch_create(fdzb_batch **out, int device);
int fdzb_batch_destroy(fdzb_batch *batch);
/* stream: a cudaStream_t; NULL = the batch's own stream. */
int fdzb_batch_set_stream(fdzb_batch *batch, void *stream);
int fdzb_batch_set_graph(fdzb_batch *batch, int enable);
/* Profiling modes as fdzb_ctx_set_profiling (FDZB_PROFILE_*). */
int fdzb_batch_set_profiling(fdzb_batch *batch, int enable);
int fdzb_batch_set_tri_order(fdzb_batch *batch, int order);
int fdzb_batch_set_occlusion_schedule(fdzb_batch *batch, int schedule);
/* fdzb_ctx_set_depth_plane for every frame of the batch's launches. */
int fdzb_batch_set_depth_plane(fdzb_batch *batch, int enable);
/* Enqueue frames[0..n) (the descriptors are copied; buffers must stay valid until
 * fdzb_batch_sync returns). */
int fdzb_batch_launch_async(fdzb_batch *batch, const fdzb_frame_desc *frames, int n);
/* Waits, re-runs the launch if the pair buffer overflowed, *ms_out (nullable)
 * gets the GPU time of the launch. */
int fdzb_batch_sync(fdzb_batch *batch, float *ms_out);
int fdzb_batch_launch(fdzb_batch *batch, const fdzb_frame_desc *frames, int n, float *ms_out);
/* Per-frame stats of the last launch (launch-wide counters read -1 when the
 * launch held more than one frame; they are in fdzb_batch_stats.totals). */
int fdzb_batch_get_frame_stats(fdzb_batch *batch, int frame, fdzb_frame_stats *out);
int fdzb_batch_get_stats(fdzb_batch *batch, fdzb_batch_stats *out);
/* Bins per side used for frame i of the last launch (>0), or an error code. */
int fdzb_batch_frame_bins(fdzb_batch *batch, int frame);
/* Bins per side and occlusion shape (see fdzb_ctx_set_occlusion_shape) used
 * for frame i of the last launch. */
int fdzb_batch_frame_shape(fdzb_batch *batch, int frame, int *bins, int *chunk, int *item);
/* An occlusion shape for every frame of later launches (0, 0: each frame's
 * tuned or default shape). */
int fdzb_batch_set_occlusion_shape(fdzb_batch *batch, int chunk, int item);
/* Open-box cull of the batch's launches (see fdzb_ctx_set_open_box). */
int fdzb_batch_set_open_box(fdzb_batch *batch, int mode);
/* Autotuner: for every size class (ceil(log2 samples), ceil(log2 triangles), N)
 * of the frames with bins == 0 not tuned yet, times three bin grids around
 * ~128 samples per bin, then at the best grid a staging chunk of 16 triangles,
 * then items of 64 samples (each candidate a launch of up to 8 copies of the
 * class's first frame, so that the GPU is as full as inside a batch) and keeps
 * the fastest grid and occlusion shape for later launches of this batch.  d_scratch: device float[scratch_floats],
 * at least one frame's W*H (receives the copies' shadows). */
int fdzb_batch_autotune(fdzb_batch *batch, const fdzb_frame_desc *frames, int n, float *d_scratch,
                        size_t scratch_floats);

/* ---- serving: a request loop with continuous batching -------------------- */

/* No counterpart in the reference (one frame per FD::FDLaunch from a
 * single-threaded GL application, FS/api.cpp:405-575).  Scenes are registered
 * once and stay resident on the device (caller-owned buffers); requests --
 * scene id, view-sample buffers, light rectangle, grid size -- are submitted
 * from any thread and return a ticket.  A worker thread owns `slots` engines
 * (stream + arena each): whenever a slot is free it launches the requests at the
 * head of the queue as one batch, as many as fit max_batch_frames,
 * max_batch_samples, max_batch_triangles and the memory budget (slot arenas -- sample and pair lists
 * -- plus the shadows and masks of the requests in flight).  Batches on
 * different slots overlap on the GPU.  Each request's results are identical to
 * a plain launch of the same inputs.  A request that does not fit the budget
 * even on an idle server completes with FDZB_ERR_NO_MEMORY. */
typedef struct fdzb_server fdzb_server;

typedef struct fdzb_serve_config {
    int32_t device;                /* < 0: current device */
    int32_t slots;                 /* concurrent batches (engines), 1..16; default 2 */
    int32_t max_batch_frames;      /* default 16 */
    int32_t use_graphs;            /* capture batches in CUDA graphs (default 0: shapes rarely repeat) */
    int64_t max_batch_samples;     /* default 16 Mi samples */
    uint64_t memory_budget_bytes;  /* default 150 GB */
    int64_t max_batch_triangles;   /* default 4 Mi triangles (bounds the batch's pair list) */
} fdzb_serve_config;

typedef struct fdzb_request {
    int32_t scene_id;
    int32_t W, H;
    int32_t bins;                  /* bins per side, power of two; 0 = autotuned / heuristic */
    const float *d_pos;            /* float4[W*H] */
    const float *d_nrm;            /* float4[W*H] */
    fdzb_area_light_desc light;
    int32_t pad0;
    float *d_shadow;               /* float[W*H] */
    uint32_t *d_masks;             /* nullable */
    const float *model_transform;  /* nullable host pointer: 16 floats applied to the scene's vertices
                                      for this request only (copied at submission) */
} fdzb_request;

typedef struct fdzb_request_result {
    int32_t status;                /* FDZB_OK or an error code */
    int32_t batch_frames;          /* requests in the launch that carried this one */
    double latency_ms;             /* submission to completion */
    double queue_ms;               /* submission to launch */
    fdzb_frame_stats stats;
} fdzb_request_result;

typedef struct fdzb_serve_stats {
    int64_t submitted, completed, rejected, failed;
    int64_t batches, batched_frames, overlapped_batches;   /* launches; frames in them; launched while another was in flight */
    int64_t queued;
    int32_t busy_slots, max_inflight_batches;
    double p50_ms, p99_ms, mean_ms, max_ms;                /* latency of completed requests */
    double frames_per_s;                                   /* completed / (last completion - first submission) */
    int64_t held_bytes, peak_bytes, budget_bytes;
    int32_t tuned_classes, slots;
} fdzb_serve_stats;

/* Fills cfg with the defaults. */
void fdzb_serve_default_config(fdzb_serve_config *cfg);
int fdzb_serve_create(fdzb_server **out, const fdzb_serve_config *cfg /* nullable: defaults */);
/* Stops the worker after the launches in flight; queued requests are dropped. */
int fdzb_serve_destroy(fdzb_server *server);
int fdzb_serve_add_scene(fdzb_server *server, const float *d_vtx, size_t n_vtx, size_t vtx_stride_bytes,
                         const int32_t *d_idx, size_t n_tri, int cull, float esp, int32_t *scene_id);
int fdzb_serve_submit(fdzb_server *server, const fdzb_request *request, uint64_t *ticket);
/* 1 = done (*out filled, ticket released), 0 = not yet, < 0 = error. */
int fdzb_serve_poll(fdzb_server *server, uint64_t ticket, fdzb_request_result *out);
/* Blocks up to timeout_ms (< 0: forever); same returns as fdzb_serve_poll. */
int fdzb_serve_wait(fdzb_server *server, uint64_t ticket, int timeout_ms, fdzb_request_result *out);
/* Waits until the queue is empty and no batch is in flight: 1, or 0 on timeout. */
int fdzb_serve_drain(fdzb_server *server, int timeout_ms);
/* Autotunes bin grids for the size classes of `requests` (see fdzb_batch_autotune);
 * call with no requests in flight. */
int fdzb_serve_autotune(fdzb_server *server, const fdzb_request *requests, int n, float *d_scratch,
                        size_t scratch_floats);
int fdzb_serve_get_stats(fdzb_server *server, fdzb_serve_stats *out);
int fdzb_serve_reset_stats(fdzb_server *server);
/* Message of the last failure inside the worker ("" if none). */
const char *fdzb_serve_last_worker_error(fdzb_server *server);

/* ---- allocation-free sort ------------------------------------------------ */

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory -- an allocator or pool that forbids cudaMalloc/cudaFree on the hot
 * path, a host process that owns every allocation, a real-time loop that may
 * not synchronise for cudaFree -- this sorts n (key, value) uint32 pairs by key,
 * stably (equal keys keep their input order), keys < key_range, using only a
 * fixed scratch area built into the library (8,917,264 bytes = 8.92 MB =
 * 8.50 MiB of device memory on every GPU that loads libfdzb.so, held until the
 * process exits).  It is the same radix sort the frame pipeline runs on its own
 * arena.
 *  - n at most FDZB_NOALLOC_SORT_MAX_PAIRS; larger n is rejected
 *    (FDZB_ERR_INVALID_ARG) before any work is enqueued;
 *  - inputs are not modified; an output that shares any byte with an input,
 *    the other output or d_status is rejected (FDZB_ERR_INVALID_ARG);
 *  - work is enqueued on `stream` (a cudaStream_t, NULL = legacy default
 *    stream) and the call returns without waiting; d_status (device int32,
 *    nullable) receives 0, or nonzero if a bounded device wait gave up;
 *  - the first call on a device looks up the scratch area's device address
 *    with cudaGetSymbolAddress, so make it before any stream capture;
 *  - every call reuses the same scratch area and clears the parts it needs
 *    (on `stream`, before its kernels); calls that overlap on the GPU (other
 *    streams or threads on the same device) race and must be ordered by the
 *    caller;
 *  - no cudaMalloc, cudaFree or other allocating routine is called. */
#define FDZB_NOALLOC_SORT_MAX_PAIRS (1 << 20)
int fdzb_sort_pairs_noalloc(const uint32_t *d_keys_in, const uint32_t *d_vals_in,
                            uint32_t *d_keys_out, uint32_t *d_vals_out, int32_t n,
                            uint32_t key_range, void *stream, int32_t *d_status);

#ifdef __cplusplus
}
#endif
#endif /* FDZB_H */
