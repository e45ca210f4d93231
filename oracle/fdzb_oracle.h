/*
 * fdzb_oracle.h -- CPU oracle for the FDZB soft-shadow path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the 4dzb_b200 package,
 * libfdzb.so) links, loads or calls this code.  It is used by tests/ as the
 * checker, by __graft_entry__.smoke() as the checker, and by bench.py for the
 * timed CPU baseline leg.
 *
 * Three oracles live here:
 *   O2  orc_frame()           FP32 restatement of the reference pipeline, stage by
 *                             stage (light setup, rectangles, light plane, triangle
 *                             setup, sample keys, stable sort, segments, bin stats,
 *                             triangle/bin pairs, per-sample occlusion, popcount).
 *                             Built with -ffp-contract=off: every + - * / is one IEEE
 *                             binary32 operation in the reference's source order.
 *   O3  orc_exhaustive_fp64() FP64 exhaustive per-light-sample edge test with no
 *                             binning and no AABB pre-cull.
 *   CPU orc_exhaustive_fp32() the O2 per-pair arithmetic run exhaustively (every
 *                             valid sample x every valid triangle) with OpenMP: the
 *                             reported CPU baseline.
 *
 * Parity is pinned against the reference's own kernel and host source compiled
 * for the CPU (oracle/ref_emu, output in oracle/_ref/) and the golden fixtures it
 * produced (tests/golden/).
 */
#ifndef FDZB_ORACLE_H
#define FDZB_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same 52-byte layout as AreaLightDes (4DZB/FDZB_Soft_Shadow/AreaLightDesc.h:3-14). */
typedef struct {
    float rightRadius, topRadius;
    float position[3], viewDir[3], upDir[3];
    int32_t lightResWidth, lightResHeight;
} orc_light_desc;

/* Derived light block; mirrors AreaLight (4DZB/FDZB_Soft_Shadow/cuda/privateDefs.h:66-101). */
typedef struct {
    float rightRadius, topRadius;
    float position[3], viewDir[3], upDir[3];
    int32_t resW, resH, resNum;
    uint32_t fullBits;
    float rightDir[3], topDir[3], x_delt[3], y_delt[3];
    float upRight[3], downLeft[3], upLeft[3], downRight[3];
    float mat[16];
    float RF[2];
    /* light grid as the occlusion stage sees it: rows along x_delt (resW of them),
     * columns along y_delt (resH); bit r * resH + c of a sample's mask */
    uint64_t fullRows, fullCols;
} orc_light;

typedef struct {
    int32_t W, H;
    const float *pos, *nrm;      /* float4[W*H], row-major, NaN x = background */
    const float *vtx;            /* vertex buffer, vtx_stride_floats floats per vertex, xyz first */
    int32_t vtx_stride_floats, V;
    const int32_t *idx;          /* int3[T] */
    int32_t T;
    int32_t bins;                /* light-plane bins per side (power of two) */
    int32_t cull;                /* triangle back-face cull */
    float esp;
    const orc_light *light;
    int32_t nthreads;            /* <= 0: OpenMP default */
    int32_t occ_stride;          /* occlusion only for sorted samples k with k % occ_stride == 0
                                    (<= 1: all); others keep mask 0 / shadow 0 */
    int32_t setup_only;          /* 1: stop after the light plane (A1-A5); enough for the
                                    exhaustive baselines, which rebuild their triangle list */
    int32_t shadow_method;       /* 0: edge-function row masks (K/Step5_2_shadowCalPerSample.inl);
                                    1: the reference's ray-cast check (K/Step5_2_calRef.inl) */
    int32_t depth_plane;         /* 1: edge-function masks also test the triangle's own plane
                                    (light samples on Q's side of it are not occluded) for
                                    triangles that reach the light plane (min depth <= 0) or
                                    the sample's depth (max depth >= the sample's) */
} orc_frame_in;

typedef struct {
    /* scalars */
    int32_t state;               /* 0 no shadow work, 1 back-facing samples only, 2 full */
    float f, sub[2];
    float sample_aabb[6], model_aabb[6];  /* min xyz, max xyz */
    float lp_begin[3], lp_end[3], lp_factor[2];
    int32_t bins_log2, num_bins, view_log2up;
    int32_t valid_samples, valid_tris, num_pairs, pair_overflow;
    int64_t pairs_tested;        /* sample/triangle pairs that pass the AABB pre-cull */
    int64_t quirk_rows_beyond_n; /* pairs whose row filter selects rows >= N (reference UB) */
    int64_t quirk_high_bits;     /* samples whose reference mask would hold bits >= N */
    int64_t quirk_key_range;     /* samples whose bin x/y fell outside the grid */
    int64_t rows_evaluated;      /* light-grid rows evaluated (3 row masks each) */
    int64_t partial_masks;       /* row masks that needed the ceil(-D/B) threshold */
    double t_total_ms, t_occ_ms; /* wall time of the call and of the occlusion stage */
    /* arrays, caller-allocated; NULL skips the copy */
    int32_t *keys, *vals;                     /* [S] position order */
    int32_t *sorted_keys, *sorted_vals;       /* [S] */
    int32_t *bin_sample_start, *bin_sample_end; /* [num_bins + 1] */
    float *bin_maxz;                          /* [num_bins] */
    float *bin_range;                         /* [4 * num_bins] */
    float *tri_aabb;                          /* [8 * T] */
    int32_t *tri_count;                       /* [T] */
    int32_t pair_capacity;
    int32_t *pair_bin, *pair_tri;             /* [pair_capacity], triangle order */
    int32_t *sorted_pair_bin, *sorted_pair_tri;
    int32_t *bin_tri_start, *bin_tri_end;     /* [num_bins] */
    uint32_t *masks;                          /* [S * words] */
    float *shadow;                            /* [S] */
} orc_frame_out;

int32_t orc_mask_words(int32_t N);
/* mask words of a rows x cols light grid (rows = lightResWidth, cols = lightResHeight) */
int32_t orc_mask_words_rc(int32_t rows, int32_t cols);
void orc_light_setup(const orc_light_desc *d, orc_light *out);
/* returns 0 on success, negative on bad input / allocation failure */
int32_t orc_frame(const orc_frame_in *in, orc_frame_out *out);

/* Exhaustive FP32 per-pair loop (CPU baseline). Samples listed in `sample_ids`
 * (row-major indices) are tested against every valid triangle.  Requires the
 * frame scalars from a previous orc_frame() call on the same inputs (`fr`).
 * Writes masks[n * words]; returns the number of pair tests executed. */
int64_t orc_exhaustive_fp32(const orc_frame_in *in, const orc_frame_out *fr,
                            const int32_t *sample_ids, int32_t n, uint32_t *masks);

/* Exhaustive FP64 per-light-sample edge test (O3).  For each listed sample,
 * every triangle of the frame (no binning, no AABB pre-cull) decides every
 * light sample in double: occluded iff all oriented edge planes (and the
 * triangle's own plane in depth-plane mode) hold, the reference's test in
 * exact arithmetic.  masks[n * words]; edge_dist[n * rows * cols] = for each
 * light sample, the distance in light-plane units (world units in the light's
 * plane) from the light sample to the boundary of the nearest triangle's
 * region seen from the sample -- inside a region the distance to its nearest
 * edge, outside the distance to the projected triangle -- exact up to
 * 1e-3 units, 1e300 where no boundary is that close (edge_dist NULL: masks
 * only, and a sample stops once all its light samples are occluded).  A conservative
 * prefilter in the light's frame skips triangles that no segment from the
 * sample to the light grid can reach; stats (nullable) counts the work. */
typedef struct {
    int64_t triangles, candidates, evaluated, fallback, skipped_blocks;
} orc_o3_stats;
void orc_exhaustive_fp64(const orc_frame_in *in, const orc_frame_out *fr,
                         const int32_t *sample_ids, int32_t n, uint32_t *masks,
                         double *edge_dist, orc_o3_stats *stats);

/* G-buffer rasteriser oracle (fdzb_raster_oracle.c): one draw. */
typedef struct {
    const float *vtx;            /* V vertices of vtx_stride_floats floats */
    int32_t vtx_stride_floats, pos_offset, nrm_offset;
    const uint32_t *idx;         /* 3 per triangle */
    int32_t n_tri;
    const int32_t *tri_material; /* nullable: material 0 */
    const float *materials;      /* 10 floats each: Ka, Kd, Ks, shininess */
    float model[16], view_proj[16];  /* column-major */
    int32_t W, H;
    int32_t clear;               /* 1: G-buffers to NaN, depth to 1 first */
} orc_raster_in;

typedef struct {
    float *g0, *g1, *g2, *g3;    /* float4[W*H] (g2, g3 nullable), row 0 = bottom */
    float *depth;                /* float[W*H] */
    int64_t sub_tris, dropped;
} orc_raster_out;

int32_t orc_raster(const orc_raster_in *in, orc_raster_out *out);

#ifdef __cplusplus
}
#endif
#endif
