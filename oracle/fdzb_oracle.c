/*
 * fdzb_oracle.c -- CPU oracle for the FDZB soft-shadow path.
 *
 * TEST INFRASTRUCTURE ONLY (see fdzb_oracle.h).  Build: oracle/Makefile, flags
 * -O2 -ffp-contract=off -fno-fast-math, so each float expression below is a
 * sequence of IEEE binary32 operations in exactly the written order.
 *
 * Reference files are cited as paths inside the 4DZB project:
 *   FS/ = 4DZB/FDZB_Soft_Shadow/, K/ = 4DZB/FDZB_Soft_Shadow/cuda/.
 *
 * Deliberate, documented differences from the reference binary:
 *  - output index y*W+x (the reference writes y<<ceil(log2 W)|x, which only
 *    matches for power-of-two W; K/Step5_2_shadowCalPerSample.inl:231);
 *  - the pair writer uses the counting kernel's clamped-AABB predicate
 *    (the reference re-tests with the unclamped AABB, K/Step4_RasterizeTriangleToBin.inl:177-193);
 *  - row masks and the row filter are restricted to the N x N light grid: the
 *    reference's inverted partial masks carry bits >= N into the popcount and,
 *    when all three row filters are inverted, index rows >= N of its shared
 *    memory (K/Step5_2_shadowCalPerSample.inl:28-31,204-222).  Both events are
 *    counted (quirk_high_bits, quirk_rows_beyond_n);
 *  - a shift by >= 32 yields 0 (PTX shl semantics of the reference's device code).
 *
 * Beyond the reference's per-sample kernel (square grids, N <= 32,
 * K/Step5_2_shadowCalPerSample.inl:249-254), the same arithmetic covers
 * rectangular grids up to 64 x 64: rows r along x_delt (lightResWidth of
 * them), columns c along y_delt (lightResHeight); the row filter bounds the
 * column term with B*(cols-1) and the rows with A*(rows-1), the row masks are
 * the reference's closed form on 64-bit words (its own template instantiated
 * for U64), and for a square grid all of it reduces to the reference's
 * formulas.  Optionally (depth_plane) a fourth plane, the triangle's own,
 * keeps light samples on the sample's side of the triangle unoccluded -- the
 * test of the reference's per-bin kernel (K/Step5_2_shadowCal.inl:667-674,
 * 838) -- for triangles that reach the light plane (min depth <= 0: the
 * occluders behind the light the per-sample kernel mis-handles) or the
 * sample's depth (max depth >= the sample's, the per-bin kernel's own
 * condition).  A triangle strictly between the light plane and the sample
 * needs no such test: the segment from the sample to any light sample in its
 * edge cone crosses it.
 */
#include "fdzb_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define F32_MAX 3.402823466e+38f

typedef struct { float x, y, z; } v3;

static inline v3 mk3(float x, float y, float z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline v3 ld3(const float *p) { return mk3(p[0], p[1], p[2]); }
static inline void st3(float *p, v3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
static inline v3 add3(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub3(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul3(v3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
/* float3 dot / cross with the component order of the CUDA-samples vector
 * helpers the reference includes (helper_math.h, not vendored): dot is
 * ((ax*bx)+(ay*by))+(az*bz); cross is (ay*bz-az*by, az*bx-ax*bz, ax*by-ay*bx). */
static inline float dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross3(v3 a, v3 b)
{
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
/* host normalize: v * (1/sqrtf(dot(v,v))) (helper_math host rsqrtf, and glm's
 * inversesqrt in 4DZB/glm/detail/func_exponential.inl:130-133). */
static inline v3 norm3(v3 v)
{
    float inv = 1.0f / sqrtf(dot3(v, v));
    return mul3(v, inv);
}

int32_t orc_mask_words(int32_t N) { return (N * N + 31) / 32; }
int32_t orc_mask_words_rc(int32_t rows, int32_t cols) { return (rows * cols + 31) / 32; }

static inline uint64_t low_bits64(int n) { return n >= 64 ? ~(uint64_t)0 : (((uint64_t)1 << n) - 1u); }

/* ---------------------------------------------------------------------------
 * A1 light setup: FS/api.cpp:303-400 (FDsetAreaLight) with GLM 0.9.8 lookAtRH
 * (4DZB/glm/gtc/matrix_transform.inl:521-546), infinitePerspectiveRH (:378-393)
 * and mat4*mat4 (4DZB/glm/detail/type_mat4x4.inl:595-614).
 * ------------------------------------------------------------------------- */
void orc_light_setup(const orc_light_desc *d, orc_light *L)
{
    memset(L, 0, sizeof(*L));
    L->rightRadius = d->rightRadius;
    L->topRadius = d->topRadius;
    memcpy(L->position, d->position, sizeof(L->position));
    L->resW = d->lightResWidth;
    L->resH = d->lightResHeight;
    L->resNum = d->lightResWidth * d->lightResHeight;
    L->fullBits = d->lightResWidth >= 32 ? 0xFFFFFFFFu : ((1u << d->lightResWidth) - 1u);
    L->fullRows = low_bits64(d->lightResWidth);
    L->fullCols = low_bits64(d->lightResHeight);

    v3 pos = ld3(d->position);
    v3 up = norm3(ld3(d->upDir));
    v3 view = norm3(ld3(d->viewDir));
    v3 right = norm3(cross3(view, up));
    v3 top = norm3(cross3(right, view));
    st3(L->upDir, up);
    st3(L->viewDir, view);
    st3(L->rightDir, right);
    st3(L->topDir, top);

    float rR = d->rightRadius, tR = d->topRadius;
    v3 xd = mul3(right, rR * -2.0f / (float)d->lightResWidth);
    v3 yd = mul3(top, tR * -2.0f / (float)d->lightResHeight);
    st3(L->x_delt, xd);
    st3(L->y_delt, yd);

    float xf = ((float)d->lightResWidth - 1.0f) / (float)d->lightResWidth;
    float yf = ((float)d->lightResHeight - 1.0f) / (float)d->lightResHeight;
    v3 nright = mul3(right, -1.0f), ntop = mul3(top, -1.0f);
    v3 ur = add3(add3(pos, mul3(mul3(right, xf), rR)), mul3(mul3(top, yf), tR));
    v3 ul = add3(add3(pos, mul3(mul3(nright, xf), rR)), mul3(mul3(top, yf), tR));
    v3 dl = add3(add3(pos, mul3(mul3(nright, xf), rR)), mul3(mul3(ntop, yf), tR));
    v3 dr = add3(add3(pos, mul3(mul3(right, xf), rR)), mul3(mul3(ntop, yf), tR));
    st3(L->upRight, ur);
    st3(L->upLeft, ul);
    st3(L->downLeft, dl);
    st3(L->downRight, dr);

    /* lookAtRH(eye = ur, center = ur + 10*view, up) */
    v3 center = add3(ur, mk3(10.0f * view.x, 10.0f * view.y, 10.0f * view.z));
    v3 fw = norm3(sub3(center, ur));
    v3 s = norm3(cross3(fw, up));
    v3 u = cross3(s, fw);
    float MV[4][4]; /* [column][row] */
    memset(MV, 0, sizeof(MV));
    MV[0][0] = 1.0f; MV[1][1] = 1.0f; MV[2][2] = 1.0f; MV[3][3] = 1.0f;
    MV[0][0] = s.x; MV[1][0] = s.y; MV[2][0] = s.z;
    MV[0][1] = u.x; MV[1][1] = u.y; MV[2][1] = u.z;
    MV[0][2] = -fw.x; MV[1][2] = -fw.y; MV[2][2] = -fw.z;
    MV[3][0] = -dot3(s, ur);
    MV[3][1] = -dot3(u, ur);
    MV[3][2] = dot3(fw, ur);

    /* infinitePerspectiveRH(120 [radians], 1, 0.1) */
    /* tan(fovy/2) correctly rounded to binary32 (double evaluation); glibc's
     * tanf(60.0f) is one ulp away from it. */
    float fovy = 120.0f, aspect = 1.0f, zNear = 0.1f;
    float range = (float)tan((double)(fovy / 2.0f)) * zNear;
    float left = -range * aspect, rightp = range * aspect, bottom = -range, topp = range;
    float P[4][4];
    memset(P, 0, sizeof(P));
    P[0][0] = (2.0f * zNear) / (rightp - left);
    P[1][1] = (2.0f * zNear) / (topp - bottom);
    P[2][2] = -1.0f;
    P[2][3] = -1.0f;
    P[3][2] = -2.0f * zNear;

    /* Result[c] = ((P0*MV[c][0] + P1*MV[c][1]) + P2*MV[c][2]) + P3*MV[c][3] */
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) {
            float a0 = P[0][r] * MV[c][0];
            float a1 = P[1][r] * MV[c][1];
            float a2 = P[2][r] * MV[c][2];
            float a3 = P[3][r] * MV[c][3];
            L->mat[c * 4 + r] = ((a0 + a1) + a2) + a3;
        }
    L->RF[0] = rR * 2.0f * xf * P[0][0] * 0.5f;
    L->RF[1] = tR * 2.0f * yf * P[1][1] * 0.5f;
}

/* K/FDprojection.inl:6-19 */
static inline v3 make_rect(const float *M, v3 t)
{
    v3 r;
    r.z = M[3] * t.x + M[7] * t.y + M[11] * t.z + M[15] * 1.0f;
    r.x = M[0] * t.x + M[4] * t.y + M[8] * t.z + M[12] * 1.0f;
    r.x = r.x / r.z * 0.5f + 0.5f;
    r.y = M[1] * t.x + M[5] * t.y + M[9] * t.z + M[13] * 1.0f;
    r.y = r.y / r.z * 0.5f + 0.5f;
    return r;
}
static inline float get_z(const float *M, v3 t)
{
    return M[3] * t.x + M[7] * t.y + M[11] * t.z + M[15] * 1.0f;
}

/* K/Step5_2_shadowCal.inl:213-222 */
static inline int point_in_tri(v3 A, v3 B, v3 C, v3 P)
{
    v3 N1 = cross3(sub3(B, A), sub3(P, B));
    v3 N2 = cross3(sub3(C, B), sub3(P, C));
    if (dot3(N1, N2) < 0.0f) return 0;
    v3 N3 = cross3(sub3(A, C), sub3(P, A));
    if (dot3(N2, N3) < 0.0f) return 0;
    return 1;
}

/* K/Step5_2_shadowCalPerSample.inl:2-12 */
static inline void plane_disc(float *A, float *B, float *C, v3 a, v3 b, v3 Q, v3 t0, v3 t1, v3 L0Q)
{
    v3 n = cross3(sub3(b, Q), sub3(a, b));
    *A = dot3(n, t0);
    *B = dot3(n, t1);
    *C = dot3(n, L0Q);
}

/* float -> int32 with PTX cvt.rzi.s32.f32 saturation (NaN -> 0). */
static inline int f2i_sat(float q)
{
    if (q != q) return 0;
    if (q >= 2147483648.0f) return 2147483647;
    if (q <= -2147483648.0f) return (int)0x80000000;
    return (int)q;
}

/* K/Step5_2_shadowCalPerSample.inl:14-33, unmasked (bits >= N may be set), on a
 * `bits`-wide word: 32 is the reference's U32, 64 its template's U64 form.  The
 * shift has PTX shl semantics: amounts >= the width (or negative) give 0. */
static _Thread_local int64_t tl_partial = 0, tl_rows = 0;

static inline uint64_t row_mask_raw(float D, float s, unsigned nm1, uint64_t full, int bits)
{
    int f1 = (D >= 0.0f);
    int f2 = (s * (float)nm1 + D >= 0.0f);
    if (f1 && f2) return full;
    if (!f1 && !f2) return 0u;
    ++tl_partial;
    float q = (-1.0f * D) / s;
    int k = f2i_sat(ceilf(q));
    uint64_t m = ((unsigned)k >= (unsigned)bits) ? 0u : ((uint64_t)1 << k);
    m -= 1u;
    if (!f1) m = ~m;
    if (bits == 32) m &= 0xFFFFFFFFu;
    return m;
}

typedef struct {
    float v0[3], v1[3], v2[3];
    float maxz, minz;
    float bmin[2], bmax[2];
} tri_rec; /* TriangleData, K/privateDefs.h:44-54 */

typedef struct {
    float ur[3], xd[3], yd[3];
    int NR, NC;              /* rows along x_delt, columns along y_delt */
    int bits;                /* row word width: 32 when both fit, else 64 */
    uint64_t fullr, fullc;   /* NR and NC low bits */
    float esp;
    int depth;               /* test the triangle's own plane too */
} pair_ctx;

static void pair_ctx_init(pair_ctx *c, const orc_light *L, float esp, int depth)
{
    memcpy(c->ur, L->upRight, sizeof(c->ur));
    memcpy(c->xd, L->x_delt, sizeof(c->xd));
    memcpy(c->yd, L->y_delt, sizeof(c->yd));
    c->NR = L->resW;
    c->NC = L->resH;
    c->bits = (L->resW <= 32 && L->resH <= 32) ? 32 : 64;
    c->fullr = L->fullRows;
    c->fullc = L->fullCols;
    c->esp = esp;
    c->depth = depth;
}

/* Ray-cast check of one sample/triangle pair (K/Step5_2_calRef.inl:1-126): for
 * every light sample not yet set, the ray from Q to the light sample (placed at
 * upRight + x_delt*j + y_delt*i, FS/api.cpp:351-357) against the triangle with
 * intersect_triangle_branchless (1e-3 < t < dist, barycentric test).  Light
 * sample (i along the height, j along the width) is stored at row j, column i,
 * the edge-function masks' layout.  The caller applies the pre-cull. */
static inline void raycast_test(const pair_ctx *c, v3 Q, const tri_rec *t, uint64_t *mask, uint64_t *full_rows)
{
    v3 p0 = ld3(t->v0), p1 = ld3(t->v1), p2 = ld3(t->v2);
    v3 e0 = sub3(p1, p0), e1 = sub3(p0, p2);
    v3 n = cross3(e1, e0);
    v3 q0 = sub3(p0, Q);
    v3 ur = ld3(c->ur), xd = ld3(c->xd), yd = ld3(c->yd);
    const float tmin = 1e-3f;
    for (int r = 0; r < c->NR; ++r) {
        if (mask[r] == c->fullc) continue;
        v3 lr = add3(ur, mul3(xd, (float)r));
        uint64_t add = 0;
        for (int col = 0; col < c->NC; ++col) {
            if (mask[r] & ((uint64_t)1 << col)) continue;
            v3 lp = add3(lr, mul3(yd, (float)col));
            v3 L = sub3(lp, Q);
            float dist = sqrtf(dot3(L, L));
            v3 dir = mk3(L.x / dist, L.y / dist, L.z / dist);
            float inv = 1.0f / dot3(n, dir);
            v3 e2 = mul3(q0, inv);
            v3 iv = cross3(dir, e2);
            float beta = dot3(iv, e1), gamma = dot3(iv, e0), tt = dot3(n, e2);
            if ((tt < dist) & (tt > tmin) & (beta >= 0.0f) & (gamma >= 0.0f) & (beta + gamma <= 1.0f))
                add |= (uint64_t)1 << col;
        }
        mask[r] |= add;
        if (mask[r] == c->fullc) *full_rows |= (uint64_t)1 << r;
    }
}

/* One sample/triangle pair: K/Step5_2_shadowCalPerSample.inl:129-222.  `mask` holds
 * NR rows of NC bits, `full_rows` the rows already full.  spZ is the sample's
 * light depth (for the depth-plane rule).  Returns 1 if the pair was evaluated
 * past the self-intersection skip.  Counters track reference quirks. */
static inline int pair_test(const pair_ctx *c, v3 Q, float spZ, const tri_rec *t, uint64_t *mask,
                            uint64_t *full_rows, int64_t *q_rows, int *q_high)
{
    v3 v0 = ld3(t->v0), v1 = ld3(t->v1), v2 = ld3(t->v2);
    v3 n = cross3(sub3(v1, v0), sub3(v2, v1));
    float dir = dot3(sub3(Q, v0), n);
    if (fabsf(dir) < c->esp && point_in_tri(v0, v1, v2, Q)) return 0;

    v3 L0 = ld3(c->ur), t0 = ld3(c->xd), t1 = ld3(c->yd);
    v3 L0Q = sub3(L0, Q);
    if (dir < 0) {
        t0 = mul3(t0, -1.0f);
        t1 = mul3(t1, -1.0f);
        L0Q = mul3(L0Q, -1.0f);
    }
    float A0, B0, C0, A1, B1, C1, A2, B2, C2;
    plane_disc(&A0, &B0, &C0, v0, v1, Q, t0, t1, L0Q);
    plane_disc(&A1, &B1, &C1, v1, v2, Q, t0, t1, L0Q);
    plane_disc(&A2, &B2, &C2, v2, v0, Q, t0, t1, L0Q);

    const unsigned nrm1 = (unsigned)(c->NR - 1), ncm1 = (unsigned)(c->NC - 1);
    const uint64_t FR = c->fullr, FC = c->fullc;
    const int bits = c->bits;
    uint64_t N0 = row_mask_raw((B0 > 0 ? B0 * (float)ncm1 : 0.0f) + C0, A0, nrm1, FR, bits);
    uint64_t N1 = row_mask_raw((B1 > 0 ? B1 * (float)ncm1 : 0.0f) + C1, A1, nrm1, FR, bits);
    uint64_t N2 = row_mask_raw((B2 > 0 ? B2 * (float)ncm1 : 0.0f) + C2, A2, nrm1, FR, bits);
    uint64_t rows = N0 & N1 & N2;
    if (rows & ~FR) ++*q_rows;
    /* the triangle's own plane: -n . (L - v0) >= 0 in the same orientation as
     * the edges, i.e. the light sample lies on the far side of the triangle */
    const int dp = c->depth && (t->minz <= 0.0f || t->maxz >= spZ);
    float A3 = 0.0f, B3 = 0.0f, C3 = 0.0f;
    if (dp) {
        v3 m = mk3(-n.x, -n.y, -n.z);
        v3 lv = sub3(L0, v0);
        if (dir < 0) lv = mul3(lv, -1.0f);
        A3 = dot3(m, t0);
        B3 = dot3(m, t1);
        C3 = dot3(m, lv);
        rows &= row_mask_raw((B3 > 0 ? B3 * (float)ncm1 : 0.0f) + C3, A3, nrm1, FR, bits);
    }
    rows &= FR & ~*full_rows;
    while (rows) {
        int r = __builtin_ctzll(rows);
        rows &= rows - 1u;
        ++tl_rows;
        uint64_t M0 = row_mask_raw(A0 * (float)r + C0, B0, ncm1, FC, bits);
        uint64_t M1 = row_mask_raw(A1 * (float)r + C1, B1, ncm1, FC, bits);
        uint64_t M2 = row_mask_raw(A2 * (float)r + C2, B2, ncm1, FC, bits);
        uint64_t m = M0 & M1 & M2;
        if (m & ~FC) *q_high = 1;
        if (dp) m &= row_mask_raw(A3 * (float)r + C3, B3, ncm1, FC, bits);
        mask[r] |= m & FC;
        if (mask[r] == FC) *full_rows |= (uint64_t)1 << r;
    }
    return 1;
}

/* rows[NR] of NC bits -> bit r * NC + c, LSB first */
static void pack_mask(const uint64_t *rows, int NR, int NC, uint32_t *out)
{
    int words = orc_mask_words_rc(NR, NC);
    memset(out, 0, sizeof(uint32_t) * words);
    for (int i = 0; i < NR; ++i)
        for (int j = 0; j < NC; ++j)
            if ((rows[i] >> j) & 1u) {
                int b = i * NC + j;
                out[b >> 5] |= 1u << (b & 31);
            }
}

static int ceil_log2_int(int v) { return (int)ceilf(log2f((float)v)); }

static double wall_s(void)
{
#ifdef _OPENMP
    return omp_get_wtime();
#else
    return 0.0;
#endif
}

/* Stable counting sort of (key, val) by key in [0, nkeys). */
static int stable_sort_pairs(const int32_t *k, const int32_t *v, int64_t n, int32_t nkeys,
                             int32_t *ko, int32_t *vo)
{
    int64_t *cnt = (int64_t *)calloc((size_t)nkeys + 1, sizeof(int64_t));
    if (!cnt) return -1;
    for (int64_t i = 0; i < n; ++i) cnt[k[i] + 1]++;
    for (int32_t i = 0; i < nkeys; ++i) cnt[i + 1] += cnt[i];
    for (int64_t i = 0; i < n; ++i) {
        int64_t p = cnt[k[i]]++;
        ko[p] = k[i];
        vo[p] = v[i];
    }
    free(cnt);
    return 0;
}

/* K/binRaster.inl:5-33 semantics: start/end for keys present, 0 elsewhere. */
static void find_start_end(const int32_t *sk, int64_t n, int32_t *start, int32_t *end, int32_t nslots)
{
    memset(start, 0, sizeof(int32_t) * nslots);
    memset(end, 0, sizeof(int32_t) * nslots);
    for (int64_t i = 0; i < n; ++i) {
        if (i == 0 || sk[i] != sk[i - 1]) {
            start[sk[i]] = (int32_t)i;
            if (i > 0) end[sk[i - 1]] = (int32_t)i;
        }
        if (i == n - 1) end[sk[i]] = (int32_t)(i + 1);
    }
}

int32_t orc_frame(const orc_frame_in *in, orc_frame_out *o)
{
    const orc_light *L = in->light;
    const float *M = L->mat;
    const int W = in->W, H = in->H, S = W * H, T = in->T, V = in->V;
    const int NR = L->resW, NC = L->resH;
    const int words = orc_mask_words_rc(NR, NC);
    if (W <= 0 || H <= 0 || NR < 1 || NR > 64 || NC < 1 || NC > 64 || in->bins < 1) return -1;
#ifdef _OPENMP
    if (in->nthreads > 0) omp_set_num_threads(in->nthreads);
#endif

    o->state = 0;
    o->valid_samples = o->valid_tris = o->num_pairs = o->pair_overflow = 0;
    o->pairs_tested = o->quirk_rows_beyond_n = o->quirk_high_bits = o->quirk_key_range = 0;
    o->rows_evaluated = o->partial_masks = 0;
    o->t_total_ms = o->t_occ_ms = 0.0;
    const double t_begin = wall_s();
    o->view_log2up = ceil_log2_int(W);
    const int log2up = o->view_log2up;
    const int Wb = in->bins, Hb = in->bins;
    o->bins_log2 = ceil_log2_int(Wb);
    o->num_bins = Wb * Hb;
    const int NB = o->num_bins;

    /* Result buffer starts cleared (FS/api.cpp:489). */
    if (o->shadow) memset(o->shadow, 0, sizeof(float) * S);
    if (o->masks) memset(o->masks, 0, sizeof(uint32_t) * (size_t)S * words);
    if (o->keys) for (int s = 0; s < S; ++s) o->keys[s] = NB;
    if (o->vals) for (int s = 0; s < S; ++s) o->vals[s] = ((s / W) << log2up) | (s % W);

    /* A3: K/Step2_1_samplerRectangleAABB.inl:1-50, K/Step2_2_modelRectangleAABB.inl:1-46 */
    float smax = -1.0f, tmax = -1.0f;
    for (int s = 0; s < S; ++s) {
        const float *p = in->pos + 4 * (size_t)s;
        if (!isnan(p[0])) smax = fmaxf(smax, get_z(M, ld3(p)));
    }
    for (int v = 0; v < V; ++v)
        tmax = fmaxf(tmax, get_z(M, ld3(in->vtx + (size_t)v * in->vtx_stride_floats)));
    if (smax < 0.0f || tmax < 0.0f) return 0;

    /* K/Step2_3_defineFDbuffer.inl:22-25 */
    float f = fmaxf(smax, tmax) + 0.1f;
    float subx = L->RF[0] / f, suby = L->RF[1] / f;
    o->f = f;
    o->sub[0] = subx;
    o->sub[1] = suby;
    o->state = 1;

    /* A4: K/Step2_1_samplerRectangleAABB.inl:53-137 */
    float *rb = (float *)malloc(sizeof(float) * 3 * (size_t)S);
    float *re = (float *)malloc(sizeof(float) * 3 * (size_t)S);
    unsigned char *backface = (unsigned char *)calloc((size_t)S, 1);
    tri_rec *rec = (tri_rec *)calloc((size_t)(T > 0 ? T : 1), sizeof(tri_rec));
    float *taabb = (float *)malloc(sizeof(float) * 8 * (size_t)(T > 0 ? T : 1));
    if (!rb || !re || !backface || !rec || !taabb) {
        free(rb); free(re); free(backface); free(rec); free(taabb);
        return -2;
    }
    v3 ur = ld3(L->upRight), ul = ld3(L->upLeft), dl = ld3(L->downLeft), dr = ld3(L->downRight);
    float sa[6] = {F32_MAX, F32_MAX, F32_MAX, -F32_MAX, -F32_MAX, -F32_MAX};
    int nvalid = 0;
    for (int s = 0; s < S; ++s) {
        const float *pp = in->pos + 4 * (size_t)s, *nn = in->nrm + 4 * (size_t)s;
        float b0 = F32_MAX, b1 = F32_MAX, b2 = F32_MAX, e0 = -F32_MAX, e1 = -F32_MAX, e2 = -F32_MAX;
        if (!isnan(pp[0])) {
            v3 p = ld3(pp), n = ld3(nn);
            if (dot3(sub3(ur, p), n) <= 0 && dot3(sub3(ul, p), n) <= 0 &&
                dot3(sub3(dl, p), n) <= 0 && dot3(sub3(dr, p), n) <= 0) {
                backface[s] = 1;
                if (o->shadow) o->shadow[s] = 1.0f;
                if (o->masks) {
                    uint64_t rows[64];
                    for (int i = 0; i < NR; ++i) rows[i] = L->fullCols;
                    pack_mask(rows, NR, NC, o->masks + (size_t)s * words);
                }
            } else {
                ++nvalid;
                v3 r = make_rect(M, p);
                b0 = r.x;
                e0 = r.x + L->RF[0] / r.z - subx;
                b1 = r.y;
                e1 = r.y + L->RF[1] / r.z - suby;
                b2 = r.z;
                e2 = r.z;
            }
        }
        rb[3 * (size_t)s] = b0; rb[3 * (size_t)s + 1] = b1; rb[3 * (size_t)s + 2] = b2;
        re[3 * (size_t)s] = e0; re[3 * (size_t)s + 1] = e1; re[3 * (size_t)s + 2] = e2;
        sa[0] = fminf(sa[0], b0); sa[1] = fminf(sa[1], b1); sa[2] = fminf(sa[2], b2);
        sa[3] = fmaxf(sa[3], e0); sa[4] = fmaxf(sa[4], e1); sa[5] = fmaxf(sa[5], e2);
    }
    memcpy(o->sample_aabb, sa, sizeof(sa));
    int ret = 0;
    if (nvalid == 0) goto done;

    /* A5: K/Step2_2_modelRectangleAABB.inl:48-99 */
    {
        float ma[6] = {F32_MAX, F32_MAX, F32_MAX, -F32_MAX, -F32_MAX, -F32_MAX};
        for (int v = 0; v < V; ++v) {
            v3 r = make_rect(M, ld3(in->vtx + (size_t)v * in->vtx_stride_floats));
            ma[0] = fminf(ma[0], r.x);
            ma[1] = fminf(ma[1], r.y);
            ma[2] = fminf(ma[2], r.z);
            ma[3] = fmaxf(ma[3], r.x + L->RF[0] / r.z - subx);
            ma[4] = fmaxf(ma[4], r.y + L->RF[1] / r.z - suby);
            ma[5] = fmaxf(ma[5], r.z);
        }
        memcpy(o->model_aabb, ma, sizeof(ma));
    }
    /* K/Step2_3_defineFDbuffer.inl:45-63 */
    if (o->model_aabb[0] > o->model_aabb[3] || o->model_aabb[1] > o->model_aabb[4] ||
        sa[0] > sa[3] || sa[1] > sa[4])
        goto done;
    float Bx = fmaxf(sa[0], o->model_aabb[0]), By = fmaxf(sa[1], o->model_aabb[1]);
    float Ex = fminf(sa[3], o->model_aabb[3]), Ey = fminf(sa[4], o->model_aabb[4]);
    o->lp_begin[0] = Bx; o->lp_begin[1] = By; o->lp_begin[2] = o->model_aabb[2];
    o->lp_end[0] = Ex; o->lp_end[1] = Ey; o->lp_end[2] = sa[5];
    if (Bx >= Ex || By >= Ey) goto done;

    /* A6: K/Step0_triangleSetup.inl:37-191 */
    {
        int nvt = 0;
        for (int t = 0; t < T; ++t) {
            const int32_t *ix = in->idx + 3 * (size_t)t;
            v3 v0 = ld3(in->vtx + (size_t)ix[0] * in->vtx_stride_floats);
            v3 v1 = ld3(in->vtx + (size_t)ix[1] * in->vtx_stride_floats);
            v3 v2 = ld3(in->vtx + (size_t)ix[2] * in->vtx_stride_floats);
            v3 e0 = sub3(v1, v0), e1 = sub3(v0, v2);
            v3 n = cross3(e1, e0);
            float mn[3] = {F32_MAX, F32_MAX, F32_MAX}, mx[3] = {-F32_MAX, -F32_MAX, -F32_MAX};
            int culled = in->cull &&
                dot3(n, sub3(ur, v0)) <= 0 && dot3(n, sub3(ur, v1)) <= 0 && dot3(n, sub3(ur, v2)) <= 0 &&
                dot3(n, sub3(ul, v0)) <= 0 && dot3(n, sub3(ul, v1)) <= 0 && dot3(n, sub3(ul, v2)) <= 0 &&
                dot3(n, sub3(dr, v0)) <= 0 && dot3(n, sub3(dr, v1)) <= 0 && dot3(n, sub3(dr, v2)) <= 0 &&
                dot3(n, sub3(dl, v0)) <= 0 && dot3(n, sub3(dl, v1)) <= 0 && dot3(n, sub3(dl, v2)) <= 0;
            if (!culled) {
                v3 vv[3] = {v0, v1, v2};
                for (int k = 0; k < 3; ++k) {
                    v3 r = make_rect(M, vv[k]);
                    mn[0] = fminf(mn[0], r.x);
                    mn[1] = fminf(mn[1], r.y);
                    mn[2] = fminf(mn[2], r.z);
                    mx[2] = fmaxf(mx[2], r.z);
                    mx[0] = fmaxf(mx[0], r.x + L->RF[0] / r.z - subx);
                    mx[1] = fmaxf(mx[1], r.y + L->RF[1] / r.z - suby);
                }
                if (!(mn[0] > Ex || mn[1] > Ey || mx[0] < Bx || mx[1] < By)) {
                    tri_rec *r = &rec[t];
                    st3(r->v0, v0); st3(r->v1, v1); st3(r->v2, v2);
                    r->minz = mn[2];
                    r->maxz = mx[2];
                    r->bmin[0] = mn[0]; r->bmin[1] = mn[1];
                    r->bmax[0] = mx[0]; r->bmax[1] = mx[1];
                    ++nvt;
                }
            }
            float *ta = taabb + 8 * (size_t)t;
            ta[0] = mn[0]; ta[1] = mn[1]; ta[2] = mn[2]; ta[3] = 1.0f;
            ta[4] = mx[0]; ta[5] = mx[1]; ta[6] = mx[2]; ta[7] = 1.0f;
        }
        o->valid_tris = nvt;
        if (o->tri_aabb) memcpy(o->tri_aabb, taabb, sizeof(float) * 8 * (size_t)T);
        if (nvt == 0) goto done;
    }

    /* K/Step2_3_defineFDbuffer.inl:99-104 */
    const int blog2 = o->bins_log2;
    const float fx = (float)Wb / (Ex - Bx), fy = (float)Hb / (Ey - By);
    o->lp_factor[0] = fx;
    o->lp_factor[1] = fy;
    o->state = 2;
    if (in->setup_only) goto done;

    /* A7: K/Step3_bindSampleToBin.inl:5-59 */
    int32_t *keys = (int32_t *)malloc(sizeof(int32_t) * (size_t)S);
    int32_t *vals = (int32_t *)malloc(sizeof(int32_t) * (size_t)S);
    int32_t *skeys = (int32_t *)malloc(sizeof(int32_t) * (size_t)S);
    int32_t *svals = (int32_t *)malloc(sizeof(int32_t) * (size_t)S);
    int32_t *sstart = (int32_t *)malloc(sizeof(int32_t) * ((size_t)NB + 1));
    int32_t *send = (int32_t *)malloc(sizeof(int32_t) * ((size_t)NB + 1));
    float *bmz = (float *)malloc(sizeof(float) * (size_t)NB);
    float *brg = (float *)malloc(sizeof(float) * 4 * (size_t)NB);
    int32_t *tcount = (int32_t *)malloc(sizeof(int32_t) * (size_t)(T > 0 ? T : 1));
    int64_t *tprefix = (int64_t *)malloc(sizeof(int64_t) * (size_t)(T > 0 ? T : 1));
    int32_t *tstart = (int32_t *)malloc(sizeof(int32_t) * (size_t)NB);
    int32_t *tend = (int32_t *)malloc(sizeof(int32_t) * (size_t)NB);
    int32_t *pbin = NULL, *ptri = NULL, *spbin = NULL, *sptri = NULL;
    if (!keys || !vals || !skeys || !svals || !sstart || !send || !bmz || !brg || !tcount ||
        !tprefix || !tstart || !tend) {
        ret = -2;
        goto free2;
    }
    {
        int nv = 0;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                size_t s = (size_t)y * W + x;
                const float *b = rb + 3 * s, *e = re + 3 * s;
                int key = NB;
                if (!((b[0] > e[0] || b[1] > e[1]) ||
                      (b[0] < Bx || b[1] < By || e[0] > Ex || e[1] > Ey))) {
                    float cx = (e[0] + b[0]) / 2.0f, cy = (e[1] + b[1]) / 2.0f;
                    int bx = (int)floorf((cx - Bx) * fx);
                    int by = (int)floorf((cy - By) * fy);
                    if (bx < 0 || bx >= Wb || by < 0 || by >= Hb) {
                        /* A centre on the far edge of the light plane rounds to bin
                         * Wb (or Hb); the reference then forms an aliased or
                         * out-of-range key.  Such samples stay unbinned here. */
                        o->quirk_key_range++;
                    } else {
                        key = (by << blog2) | bx;
                        ++nv;
                    }
                }
                keys[s] = key;
                vals[s] = (y << log2up) | x;
            }
        o->valid_samples = nv;
    }
    if (o->keys) memcpy(o->keys, keys, sizeof(int32_t) * S);

    /* A8 + A9: K/Step3_bindSampleToBin.inl:125-133, K/binRaster.inl:36-46 */
    if (stable_sort_pairs(keys, vals, S, NB + 1, skeys, svals)) { ret = -2; goto free2; }
    find_start_end(skeys, S, sstart, send, NB + 1);
    if (o->sorted_keys) memcpy(o->sorted_keys, skeys, sizeof(int32_t) * S);
    if (o->sorted_vals) memcpy(o->sorted_vals, svals, sizeof(int32_t) * S);
    if (o->bin_sample_start) memcpy(o->bin_sample_start, sstart, sizeof(int32_t) * (NB + 1));
    if (o->bin_sample_end) memcpy(o->bin_sample_end, send, sizeof(int32_t) * (NB + 1));

    /* A10: K/Step3_bindSampleToBin.inl:61-104 */
    for (int b = 0; b < NB; ++b) {
        float mz = -F32_MAX, r0 = -F32_MAX, r1 = -F32_MAX, r2 = F32_MAX, r3 = F32_MAX;
        for (int i = sstart[b]; i < send[b]; ++i) {
            int sv = svals[i];
            size_t s = (size_t)(sv >> log2up) * W + (sv & ((1 << log2up) - 1));
            mz = fmaxf(mz, rb[3 * s + 2]);
            r0 = fmaxf(r0, rb[3 * s]);
            r1 = fmaxf(r1, rb[3 * s + 1]);
            r2 = fminf(r2, re[3 * s]);
            r3 = fminf(r3, re[3 * s + 1]);
        }
        bmz[b] = mz;
        brg[4 * b] = r0; brg[4 * b + 1] = r1; brg[4 * b + 2] = r2; brg[4 * b + 3] = r3;
    }
    if (o->bin_maxz) memcpy(o->bin_maxz, bmz, sizeof(float) * NB);
    if (o->bin_range) memcpy(o->bin_range, brg, sizeof(float) * 4 * NB);

    /* A11: K/Step4_RasterizeTriangleToBin.inl:5-113 (the clamped AABB predicate is
     * used for both counting and writing). */
    int64_t total = 0;
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            int64_t cap = o->pair_capacity > total ? o->pair_capacity : total;
            pbin = (int32_t *)malloc(sizeof(int32_t) * (size_t)(cap > 0 ? cap : 1));
            ptri = (int32_t *)malloc(sizeof(int32_t) * (size_t)(cap > 0 ? cap : 1));
            spbin = (int32_t *)malloc(sizeof(int32_t) * (size_t)(cap > 0 ? cap : 1));
            sptri = (int32_t *)malloc(sizeof(int32_t) * (size_t)(cap > 0 ? cap : 1));
            if (!pbin || !ptri || !spbin || !sptri) { ret = -2; goto free2; }
        }
        for (int t = 0; t < T; ++t) {
            const float *ta = taabb + 8 * (size_t)t;
            float bx = ta[0], by = ta[1], bz = ta[2], ex = ta[4], ey = ta[5], ez = ta[6];
            int cnt = 0;
            int64_t base = pass ? tprefix[t] : 0;
            if (!(bx > ex || by > ey || bz > ez || bx > Ex || by > Ey || ex < Bx || ey < By)) {
                bx = fmaxf(bx, Bx);
                by = fmaxf(by, By);
                ex = fminf(ex, Ex);
                ey = fminf(ey, Ey);
                int cbx = (int)(unsigned short)fmaxf(floorf((bx - Bx) * fx), 0.0f);
                int cby = (int)(unsigned short)fmaxf(floorf((by - By) * fy), 0.0f);
                int cex = (int)(unsigned short)fminf(ceilf((ex - Bx) * fx), (float)Wb);
                int cey = (int)(unsigned short)fminf(ceilf((ey - By) * fy), (float)Hb);
                for (int j = cby; j < cey; ++j)
                    for (int i = cbx; i < cex; ++i) {
                        int bin = (j << blog2) | i;
                        const float *R = brg + 4 * (size_t)bin;
                        if (bmz[bin] >= bz && bx < R[0] && by < R[1] && R[2] < ex && R[3] < ey) {
                            if (pass) {
                                pbin[base + cnt] = bin;
                                ptri[base + cnt] = t;
                            }
                            ++cnt;
                        }
                    }
            }
            if (!pass) {
                tcount[t] = cnt;
                tprefix[t] = total;
                total += cnt;
            }
        }
    }
    if (o->tri_count) memcpy(o->tri_count, tcount, sizeof(int32_t) * T);
    o->num_pairs = (int32_t)total;
    o->pair_overflow = total > o->pair_capacity;
    if (o->pair_bin && !o->pair_overflow) memcpy(o->pair_bin, pbin, sizeof(int32_t) * total);
    if (o->pair_tri && !o->pair_overflow) memcpy(o->pair_tri, ptri, sizeof(int32_t) * total);

    /* A13: K/Step4_RasterizeTriangleToBin.inl:220-228, K/binRaster.inl:49-59 */
    if (stable_sort_pairs(pbin, ptri, total, NB, spbin, sptri)) { ret = -2; goto free2; }
    find_start_end(spbin, total, tstart, tend, NB);
    if (o->sorted_pair_bin && !o->pair_overflow) memcpy(o->sorted_pair_bin, spbin, sizeof(int32_t) * total);
    if (o->sorted_pair_tri && !o->pair_overflow) memcpy(o->sorted_pair_tri, sptri, sizeof(int32_t) * total);
    if (o->bin_tri_start) memcpy(o->bin_tri_start, tstart, sizeof(int32_t) * NB);
    if (o->bin_tri_end) memcpy(o->bin_tri_end, tend, sizeof(int32_t) * NB);

    /* A14 + A15: K/Step5_2_shadowCalPerSample.inl:37-231 */
    {
        const double t_occ0 = wall_s();
        pair_ctx c;
        pair_ctx_init(&c, L, in->esp, in->depth_plane);
        const int Sv = o->valid_samples;
        const int stride = in->occ_stride > 1 ? in->occ_stride : 1;
        int64_t tested = 0, qrows = 0, qhigh = 0, nrows = 0, npart = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : tested, qrows, qhigh, nrows, npart)
        for (int k = 0; k < Sv; ++k) {
            if (k % stride) continue;
            tl_rows = 0;
            tl_partial = 0;
            int sv = svals[k], bin = skeys[k];
            size_t s = (size_t)(sv >> log2up) * W + (sv & ((1 << log2up) - 1));
            v3 Q = ld3(in->pos + 4 * s);
            float spx = rb[3 * s], spy = rb[3 * s + 1], spz = re[3 * s], spw = re[3 * s + 1];
            float spZ = re[3 * s + 2];
            uint64_t rows[64];
            memset(rows, 0, sizeof(rows));
            uint64_t full_rows = 0;
            int high = 0;
            for (int p = tstart[bin]; p < tend[bin] && full_rows != c.fullr; ++p) {
                const tri_rec *t = &rec[sptri[p]];
                if (in->shadow_method == 1) {
                    /* refCal's pre-cull: rectangle containment, and the depth test
                     * with a double literal (K/Step5_2_calRef.inl:98-102) */
                    if (!(spz <= t->bmax[0] && spw <= t->bmax[1] && spx >= t->bmin[0] && spy >= t->bmin[1]))
                        continue;
                    if ((double)t->minz - 1e-3 > (double)spZ) continue;
                    ++tested;
                    raycast_test(&c, Q, t, rows, &full_rows);
                    continue;
                }
                if (!(t->bmin[0] <= spx && t->bmin[1] <= spy && spz <= t->bmax[0] &&
                      spw <= t->bmax[1] && t->minz <= spZ))
                    continue;
                ++tested;
                pair_test(&c, Q, spZ, t, rows, &full_rows, &qrows, &high);
            }
            qhigh += high;
            nrows += tl_rows;
            npart += tl_partial;
            int cnt = 0;
            for (int i = 0; i < NR; ++i) cnt += __builtin_popcountll(rows[i]);
            if (o->shadow) o->shadow[s] = (float)cnt / (float)(NR * NC);
            if (o->masks) pack_mask(rows, NR, NC, o->masks + s * words);
        }
        o->pairs_tested = tested;
        o->quirk_rows_beyond_n = qrows;
        o->quirk_high_bits = qhigh;
        o->rows_evaluated = nrows;
        o->partial_masks = npart;
        o->t_occ_ms = 1e3 * (wall_s() - t_occ0);
    }

free2:
    free(keys); free(vals); free(skeys); free(svals); free(sstart); free(send);
    free(bmz); free(brg); free(tcount); free(tprefix); free(tstart); free(tend);
    free(pbin); free(ptri); free(spbin); free(sptri);
done:
    free(rb); free(re); free(backface); free(rec); free(taabb);
    o->t_total_ms = 1e3 * (wall_s() - t_begin);
    return ret;
}

/* Valid-triangle list and records rebuilt from the frame's light-plane scalars. */
static int build_tri_list(const orc_frame_in *in, const orc_frame_out *fr, tri_rec **recs_out)
{
    const orc_light *L = in->light;
    const float *M = L->mat;
    v3 ur = ld3(L->upRight), ul = ld3(L->upLeft), dl = ld3(L->downLeft), dr = ld3(L->downRight);
    tri_rec *recs = (tri_rec *)malloc(sizeof(tri_rec) * (size_t)(in->T > 0 ? in->T : 1));
    if (!recs) return -1;
    int n = 0;
    for (int t = 0; t < in->T; ++t) {
        const int32_t *ix = in->idx + 3 * (size_t)t;
        v3 v0 = ld3(in->vtx + (size_t)ix[0] * in->vtx_stride_floats);
        v3 v1 = ld3(in->vtx + (size_t)ix[1] * in->vtx_stride_floats);
        v3 v2 = ld3(in->vtx + (size_t)ix[2] * in->vtx_stride_floats);
        v3 n3 = cross3(sub3(v0, v2), sub3(v1, v0));
        int culled = in->cull &&
            dot3(n3, sub3(ur, v0)) <= 0 && dot3(n3, sub3(ur, v1)) <= 0 && dot3(n3, sub3(ur, v2)) <= 0 &&
            dot3(n3, sub3(ul, v0)) <= 0 && dot3(n3, sub3(ul, v1)) <= 0 && dot3(n3, sub3(ul, v2)) <= 0 &&
            dot3(n3, sub3(dr, v0)) <= 0 && dot3(n3, sub3(dr, v1)) <= 0 && dot3(n3, sub3(dr, v2)) <= 0 &&
            dot3(n3, sub3(dl, v0)) <= 0 && dot3(n3, sub3(dl, v1)) <= 0 && dot3(n3, sub3(dl, v2)) <= 0;
        if (culled) continue;
        float mn[3] = {F32_MAX, F32_MAX, F32_MAX}, mx[3] = {-F32_MAX, -F32_MAX, -F32_MAX};
        v3 vv[3] = {v0, v1, v2};
        for (int k = 0; k < 3; ++k) {
            v3 r = make_rect(M, vv[k]);
            mn[0] = fminf(mn[0], r.x);
            mn[1] = fminf(mn[1], r.y);
            mn[2] = fminf(mn[2], r.z);
            mx[2] = fmaxf(mx[2], r.z);
            mx[0] = fmaxf(mx[0], r.x + L->RF[0] / r.z - fr->sub[0]);
            mx[1] = fmaxf(mx[1], r.y + L->RF[1] / r.z - fr->sub[1]);
        }
        tri_rec *r = &recs[n++];
        st3(r->v0, v0); st3(r->v1, v1); st3(r->v2, v2);
        r->minz = mn[2]; r->maxz = mx[2];
        r->bmin[0] = mn[0]; r->bmin[1] = mn[1]; r->bmax[0] = mx[0]; r->bmax[1] = mx[1];
    }
    *recs_out = recs;
    return n;
}

int64_t orc_exhaustive_fp32(const orc_frame_in *in, const orc_frame_out *fr,
                            const int32_t *sample_ids, int32_t n, uint32_t *masks)
{
    const orc_light *L = in->light;
    const int NR = L->resW, NC = L->resH, words = orc_mask_words_rc(NR, NC);
    memset(masks, 0, sizeof(uint32_t) * (size_t)n * words);
    if (fr->state < 2) return 0;
    tri_rec *recs = NULL;
    int nt = build_tri_list(in, fr, &recs);
    if (nt < 0) return -1;
    pair_ctx c;
    pair_ctx_init(&c, L, in->esp, in->depth_plane);
    const float *M = L->mat;
    const float Bx = fr->lp_begin[0], By = fr->lp_begin[1], Ex = fr->lp_end[0], Ey = fr->lp_end[1];
    v3 ur = ld3(L->upRight), ul = ld3(L->upLeft), dl = ld3(L->downLeft), dr = ld3(L->downRight);
#ifdef _OPENMP
    if (in->nthreads > 0) omp_set_num_threads(in->nthreads);
#endif
    int64_t tested = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : tested)
    for (int k = 0; k < n; ++k) {
        size_t s = (size_t)sample_ids[k];
        const float *pp = in->pos + 4 * s, *nn = in->nrm + 4 * s;
        if (isnan(pp[0])) continue;
        v3 p = ld3(pp), nv = ld3(nn);
        if (dot3(sub3(ur, p), nv) <= 0 && dot3(sub3(ul, p), nv) <= 0 &&
            dot3(sub3(dl, p), nv) <= 0 && dot3(sub3(dr, p), nv) <= 0) {
            uint64_t rows[64];
            for (int i = 0; i < NR; ++i) rows[i] = c.fullc;
            pack_mask(rows, NR, NC, masks + (size_t)k * words);
            continue;
        }
        v3 r = make_rect(M, p);
        float spx = r.x, spy = r.y;
        float spz = r.x + L->RF[0] / r.z - fr->sub[0], spw = r.y + L->RF[1] / r.z - fr->sub[1];
        float spZ = r.z;
        /* same validity as the sample key pass, K/Step3_bindSampleToBin.inl:35-38 */
        if ((spx > spz || spy > spw) || (spx < Bx || spy < By || spz > Ex || spw > Ey)) continue;
        uint64_t rows[64];
        memset(rows, 0, sizeof(rows));
        uint64_t full_rows = 0;
        int64_t qr = 0;
        int hi = 0;
        for (int t = 0; t < nt && full_rows != c.fullr; ++t) {
            const tri_rec *tr = &recs[t];
            if (!(tr->bmin[0] <= spx && tr->bmin[1] <= spy && spz <= tr->bmax[0] &&
                  spw <= tr->bmax[1] && tr->minz <= spZ))
                continue;
            ++tested;
            pair_test(&c, p, spZ, tr, rows, &full_rows, &qr, &hi);
        }
        pack_mask(rows, NR, NC, masks + (size_t)k * words);
    }
    free(recs);
    return tested;
}

/* O3: FP64 exhaustive per-light-sample test.  Same sample validity, same
 * triangle set (FP32 back-face predicate), same orientation and self-skip rules;
 * every light sample (i, j) at L0 + i*x_delt + j*y_delt (i < resW, j < resH) is
 * occluded iff all three oriented edge functions are >= 0 -- with depth_plane,
 * and the triangle's max depth not below the sample's, also the oriented
 * triangle plane -- evaluated in double. */
/* ---- O3: FP64 per-light-sample test ------------------------------------
 *
 * Light frame, in double: origin upRight, axes x_delt and y_delt (one light
 * sample per unit: light sample (i, j) sits at a = i, b = j, d = 0) and the unit
 * normal nv of the light plane, oriented along viewDir (towards the
 * receivers).  (a, b, d) of a point P solve P - upRight = a x_delt + b y_delt +
 * d nv.  Light-plane units are world units measured in the light's plane:
 * a grid step along x_delt is |x_delt| of them. */
typedef struct {
    double o[3], inv[3][3];
    double sx, sy;
} o3_frame;

static void o3_frame_init(o3_frame *F, const orc_light *L)
{
    double X[3], Y[3], N[3];
    for (int k = 0; k < 3; ++k) {
        F->o[k] = L->upRight[k];
        X[k] = L->x_delt[k];
        Y[k] = L->y_delt[k];
    }
    N[0] = X[1] * Y[2] - X[2] * Y[1];
    N[1] = X[2] * Y[0] - X[0] * Y[2];
    N[2] = X[0] * Y[1] - X[1] * Y[0];
    double nn = sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
    double sg = (N[0] * L->viewDir[0] + N[1] * L->viewDir[1] + N[2] * L->viewDir[2]) < 0 ? -1.0 : 1.0;
    for (int k = 0; k < 3; ++k) N[k] *= sg / nn;
    /* inverse of the column matrix [X Y N] by cofactors */
    double m[3][3] = {{X[0], Y[0], N[0]}, {X[1], Y[1], N[1]}, {X[2], Y[2], N[2]}};
    double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
                 m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                 m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            int r1 = (c + 1) % 3, r2 = (c + 2) % 3, c1 = (r + 1) % 3, c2 = (r + 2) % 3;
            F->inv[r][c] = (m[r1][c1] * m[r2][c2] - m[r1][c2] * m[r2][c1]) / det;
        }
    F->sx = sqrt(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
    F->sy = sqrt(Y[0] * Y[0] + Y[1] * Y[1] + Y[2] * Y[2]);
}

static inline void o3_coords(const o3_frame *F, const double P[3], double out[3])
{
    double q[3] = {P[0] - F->o[0], P[1] - F->o[1], P[2] - F->o[2]};
    for (int r = 0; r < 3; ++r) out[r] = F->inv[r][0] * q[0] + F->inv[r][1] * q[1] + F->inv[r][2] * q[2];
}

/* Triangles are visited in blocks of O3_BLOCK, spatially sorted, each block
 * with the union of its members' frame bounds, so that one test skips a block
 * that no segment from the sample to the light grid can reach. */
#define O3_BLOCK 64
/* Boundary distances are exact up to this many light-plane units; a light
 * sample farther from every triangle's projected boundary keeps 1e300. */
#define O3_MARGIN 1e-3

typedef struct {
    double lo[3], hi[3];   /* frame bounds (a, b, d) */
} o3_box;

/* Can a segment from a light sample of the [0, NR-1] x [0, NC-1] grid to the
 * point q = (aQ, bQ, dQ) meet a point of box B?  A point at depth d of such a
 * segment is (1 - s) (i, j, 0) + s q with s = d / dQ, so over the box's depth
 * range its (a, b) lie in the hull of the grid's images at the two end values
 * of s (the images are intervals whose ends move linearly in s).  The test
 * widens them by mg grid units.  Conservative: false only when no segment can
 * meet the box.  The cone test extends the segments beyond the light plane
 * (d < 0, s < 0), which this covers too. */
static inline int o3_reach(const o3_box *B, const double q[3], int NR, int NC, double mg)
{
    if (B->lo[2] >= q[2]) return 0;    /* at or behind the sample's depth */
    double s0 = B->lo[2] / q[2], s1 = B->hi[2] / q[2];
    if (s1 > 1.0) s1 = 1.0;
    for (int ax = 0; ax < 2; ++ax) {
        double ext = ax == 0 ? (double)(NR - 1) : (double)(NC - 1);
        double l0 = s0 * q[ax], l1 = s1 * q[ax];
        double h0 = (1.0 - s0) * ext + l0, h1 = (1.0 - s1) * ext + l1;
        double lo = (l0 < l1 ? l0 : l1) - mg, hi = (h0 > h1 ? h0 : h1) + mg;
        if (B->hi[ax] < lo || B->lo[ax] > hi) return 0;
    }
    return 1;
}

static uint32_t o3_morton(uint32_t x, uint32_t y, uint32_t z)
{
    uint32_t r = 0;
    for (int k = 0; k < 10; ++k)
        r |= ((x >> k) & 1u) << (3 * k) | ((y >> k) & 1u) << (3 * k + 1) | ((z >> k) & 1u) << (3 * k + 2);
    return r;
}

typedef struct {
    double key;
    int blk;
} o3_visit;

static int o3_cmp_visit(const void *a, const void *b)
{
    const o3_visit *x = (const o3_visit *)a, *y = (const o3_visit *)b;
    return x->key > y->key ? -1 : x->key < y->key ? 1 : x->blk - y->blk;
}

static const uint32_t *o3_sort_keys;
static int o3_cmp(const void *a, const void *b)
{
    uint32_t x = o3_sort_keys[*(const int *)a], y = o3_sort_keys[*(const int *)b];
    return x < y ? -1 : x > y ? 1 : (*(const int *)a - *(const int *)b);
}

static inline double o3_seg_dist(double px, double py, const double a[2], const double b[2])
{
    double dx = b[0] - a[0], dy = b[1] - a[1];
    double L2 = dx * dx + dy * dy;
    double t = L2 > 0 ? ((px - a[0]) * dx + (py - a[1]) * dy) / L2 : 0.0;
    if (t < 0) t = 0;
    if (t > 1) t = 1;
    double ex = a[0] + t * dx - px, ey = a[1] + t * dy - py;
    return sqrt(ex * ex + ey * ey);
}

void orc_exhaustive_fp64(const orc_frame_in *in, const orc_frame_out *fr,
                         const int32_t *sample_ids, int32_t n, uint32_t *masks,
                         double *edge_dist, orc_o3_stats *stats)
{
    const orc_light *L = in->light;
    const int NR = L->resW, NC = L->resH, words = orc_mask_words_rc(NR, NC), NN = NR * NC;
    memset(masks, 0, sizeof(uint32_t) * (size_t)n * words);
    if (edge_dist)
        for (size_t i = 0; i < (size_t)n * NN; ++i) edge_dist[i] = 1e300;
    if (stats) memset(stats, 0, sizeof(*stats));
    if (fr->state < 2) return;
    tri_rec *recs = NULL;
    int nt = build_tri_list(in, fr, &recs);
    if (nt < 0) return;
    /* without distances a sample stops once every light sample is occluded:
     * the mask is an OR over triangles and can gain nothing more */
    const int need_dist = edge_dist != NULL;
    o3_frame F;
    o3_frame_init(&F, L);
    const double mg = O3_MARGIN / (F.sx < F.sy ? F.sx : F.sy);
    /* frame coordinates of every vertex; spatial order; block bounds */
    double *fv = (double *)malloc(sizeof(double) * 9 * (size_t)(nt > 0 ? nt : 1));
    o3_box *tb = (o3_box *)malloc(sizeof(o3_box) * (size_t)(nt > 0 ? nt : 1));
    uint32_t *key = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(nt > 0 ? nt : 1));
    int *order = (int *)malloc(sizeof(int) * (size_t)(nt > 0 ? nt : 1));
    const int nblk = (nt + O3_BLOCK - 1) / O3_BLOCK;
    o3_box *bb = (o3_box *)malloc(sizeof(o3_box) * (size_t)(nblk > 0 ? nblk : 1));
    if (!fv || !tb || !key || !order || !bb) {
        free(fv); free(tb); free(key); free(order); free(bb); free(recs);
        return;
    }
    double glo[3] = {1e300, 1e300, 1e300}, ghi[3] = {-1e300, -1e300, -1e300};
    for (int t = 0; t < nt; ++t) {
        const float *vs[3] = {recs[t].v0, recs[t].v1, recs[t].v2};
        o3_box *B = &tb[t];
        for (int k = 0; k < 3; ++k) {
            B->lo[k] = 1e300;
            B->hi[k] = -1e300;
        }
        for (int v = 0; v < 3; ++v) {
            double P[3] = {vs[v][0], vs[v][1], vs[v][2]};
            double *c = fv + 9 * (size_t)t + 3 * v;
            o3_coords(&F, P, c);
            for (int k = 0; k < 3; ++k) {
                if (c[k] < B->lo[k]) B->lo[k] = c[k];
                if (c[k] > B->hi[k]) B->hi[k] = c[k];
            }
        }
        for (int k = 0; k < 3; ++k) {
            double mid = 0.5 * (B->lo[k] + B->hi[k]);
            if (mid < glo[k]) glo[k] = mid;
            if (mid > ghi[k]) ghi[k] = mid;
        }
    }
    for (int t = 0; t < nt; ++t) {
        uint32_t q[3];
        for (int k = 0; k < 3; ++k) {
            double mid = 0.5 * (tb[t].lo[k] + tb[t].hi[k]);
            double u = ghi[k] > glo[k] ? (mid - glo[k]) / (ghi[k] - glo[k]) : 0.0;
            q[k] = (uint32_t)(u * 1023.0 + 0.5);
        }
        key[t] = o3_morton(q[0], q[1], q[2]);
        order[t] = t;
    }
    o3_sort_keys = key;
    qsort(order, (size_t)nt, sizeof(int), o3_cmp);
    for (int b = 0; b < nblk; ++b) {
        o3_box *B = &bb[b];
        for (int k = 0; k < 3; ++k) {
            B->lo[k] = 1e300;
            B->hi[k] = -1e300;
        }
        for (int m = b * O3_BLOCK; m < nt && m < (b + 1) * O3_BLOCK; ++m)
            for (int k = 0; k < 3; ++k) {
                if (tb[order[m]].lo[k] < B->lo[k]) B->lo[k] = tb[order[m]].lo[k];
                if (tb[order[m]].hi[k] > B->hi[k]) B->hi[k] = tb[order[m]].hi[k];
            }
    }

    const float *M = L->mat;
    const float Bx = fr->lp_begin[0], By = fr->lp_begin[1], Ex = fr->lp_end[0], Ey = fr->lp_end[1];
    v3 ur = ld3(L->upRight), ul = ld3(L->upLeft), dl = ld3(L->downLeft), dr = ld3(L->downRight);
    const double L0[3] = {L->upRight[0], L->upRight[1], L->upRight[2]};
    const double XD[3] = {L->x_delt[0], L->x_delt[1], L->x_delt[2]};
    const double YD[3] = {L->y_delt[0], L->y_delt[1], L->y_delt[2]};
    const double desp = in->esp, sx = F.sx, sy = F.sy;
    int64_t cand = 0, evald = 0, fallback = 0, skipped_blocks = 0;
#ifdef _OPENMP
    if (in->nthreads > 0) omp_set_num_threads(in->nthreads);
#endif
#pragma omp parallel reduction(+ : cand, evald, fallback, skipped_blocks)
    {
    /* reachable blocks of a sample, deepest (nearest the receivers, the
     * largest seen from the sample) first, so that a sample in umbra fills
     * its mask early when distances are not asked for */
    o3_visit *visit = (o3_visit *)malloc(sizeof(o3_visit) * (size_t)(nblk > 0 ? nblk : 1));
#pragma omp for schedule(dynamic, 4)
    for (int k = 0; k < n; ++k) {
        size_t s = (size_t)sample_ids[k];
        const float *pp = in->pos + 4 * s, *nn = in->nrm + 4 * s;
        uint32_t *mk = masks + (size_t)k * words;
        double *ed = need_dist ? edge_dist + (size_t)k * NN : NULL;
        int nset = 0;
        if (isnan(pp[0])) continue;
        v3 p = ld3(pp), nv = ld3(nn);
        if (dot3(sub3(ur, p), nv) <= 0 && dot3(sub3(ul, p), nv) <= 0 &&
            dot3(sub3(dl, p), nv) <= 0 && dot3(sub3(dr, p), nv) <= 0) {
            for (int b = 0; b < NN; ++b) mk[b >> 5] |= 1u << (b & 31);
            continue;
        }
        v3 r = make_rect(M, p);
        if (r.x < Bx || r.y < By || r.x + L->RF[0] / r.z - fr->sub[0] > Ex ||
            r.y + L->RF[1] / r.z - fr->sub[1] > Ey)
            continue;
        const double Q[3] = {p.x, p.y, p.z};
        double q[3];
        o3_coords(&F, Q, q);
        const int prefilter = q[2] > 0;   /* the sample in front of the light plane */
        int nvisit = 0;
        for (int blk = 0; blk < nblk; ++blk) {
            if (prefilter && !o3_reach(&bb[blk], q, NR, NC, mg)) {
                ++skipped_blocks;
                continue;
            }
            visit[nvisit].key = bb[blk].hi[2];
            visit[nvisit].blk = blk;
            ++nvisit;
        }
        qsort(visit, (size_t)nvisit, sizeof(o3_visit), o3_cmp_visit);
        for (int vi = 0; vi < nvisit && (need_dist || nset < NN); ++vi) {
            const int blk = visit[vi].blk;
            for (int m = blk * O3_BLOCK; m < nt && m < (blk + 1) * O3_BLOCK && (need_dist || nset < NN); ++m) {
                const int t = order[m];
                if (prefilter && !o3_reach(&tb[t], q, NR, NC, mg)) continue;
                ++cand;
                const tri_rec *tr = &recs[t];
                double V[3][3];
                for (int a = 0; a < 3; ++a) {
                    V[0][a] = tr->v0[a];
                    V[1][a] = tr->v1[a];
                    V[2][a] = tr->v2[a];
                }
                double e1[3], e2[3], nrm[3], qv[3];
                for (int a = 0; a < 3; ++a) {
                    e1[a] = V[1][a] - V[0][a];
                    e2[a] = V[2][a] - V[1][a];
                    qv[a] = Q[a] - V[0][a];
                }
                nrm[0] = e1[1] * e2[2] - e1[2] * e2[1];
                nrm[1] = e1[2] * e2[0] - e1[0] * e2[2];
                nrm[2] = e1[0] * e2[1] - e1[1] * e2[0];
                double dir = qv[0] * nrm[0] + qv[1] * nrm[1] + qv[2] * nrm[2];
                if (fabs(dir) < desp) {
                    /* point-in-triangle in double, K/Step5_2_shadowCal.inl:213-222 */
                    double Nv[3][3];
                    for (int e = 0; e < 3; ++e) {
                        const double *A = V[e], *B = V[(e + 1) % 3];
                        double ba[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
                        double pb[3] = {Q[0] - B[0], Q[1] - B[1], Q[2] - B[2]};
                        Nv[e][0] = ba[1] * pb[2] - ba[2] * pb[1];
                        Nv[e][1] = ba[2] * pb[0] - ba[0] * pb[2];
                        Nv[e][2] = ba[0] * pb[1] - ba[1] * pb[0];
                    }
                    double d12 = Nv[0][0] * Nv[1][0] + Nv[0][1] * Nv[1][1] + Nv[0][2] * Nv[1][2];
                    double d23 = Nv[1][0] * Nv[2][0] + Nv[1][1] * Nv[2][1] + Nv[1][2] * Nv[2][2];
                    if (!(d12 < 0.0) && !(d23 < 0.0)) continue;
                }
                double sg = dir < 0 ? -1.0 : 1.0;
                double A[4], B[4], C[4], inv[4], pn[4];
                const int planes = (in->depth_plane && (tr->minz <= 0.0f || tr->maxz >= r.z)) ? 4 : 3;
                for (int e = 0; e < 3; ++e) {
                    const double *a = V[e], *b = V[(e + 1) % 3];
                    double u[3] = {b[0] - Q[0], b[1] - Q[1], b[2] - Q[2]};
                    double w[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
                    double nk[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
                    double lq[3] = {L0[0] - Q[0], L0[1] - Q[1], L0[2] - Q[2]};
                    A[e] = sg * (nk[0] * XD[0] + nk[1] * XD[1] + nk[2] * XD[2]);
                    B[e] = sg * (nk[0] * YD[0] + nk[1] * YD[1] + nk[2] * YD[2]);
                    C[e] = sg * (nk[0] * lq[0] + nk[1] * lq[1] + nk[2] * lq[2]);
                }
                if (planes == 4) {
                    /* -n . (L - v0), oriented like the edges */
                    double lv[3] = {L0[0] - V[0][0], L0[1] - V[0][1], L0[2] - V[0][2]};
                    A[3] = -sg * (nrm[0] * XD[0] + nrm[1] * XD[1] + nrm[2] * XD[2]);
                    B[3] = -sg * (nrm[0] * YD[0] + nrm[1] * YD[1] + nrm[2] * YD[2]);
                    C[3] = -sg * (nrm[0] * lv[0] + nrm[1] * lv[1] + nrm[2] * lv[2]);
                }
                for (int e = 0; e < planes; ++e) {
                    double g = sqrt(A[e] * A[e] + B[e] * B[e]);
                    inv[e] = g > 0 ? 1.0 / g : 1e300;
                    /* light-plane units per unit of A i + B j + C */
                    double h = sqrt((A[e] / sx) * (A[e] / sx) + (B[e] / sy) * (B[e] / sy));
                    pn[e] = h > 0 ? 1.0 / h : 1e300;
                }
                /* the triangle seen from Q on the light plane: each vertex
                 * closer to the light than Q projects at q + t (v - q),
                 * t = dQ / (dQ - dv) > 0 */
                int proj = planes == 3 && prefilter;
                double pv[3][2];
                for (int v = 0; v < 3 && proj; ++v) {
                    const double *c = fv + 9 * (size_t)t + 3 * v;
                    if (!(c[2] < q[2])) {
                        proj = 0;
                        break;
                    }
                    double tt = q[2] / (q[2] - c[2]);
                    pv[v][0] = q[0] + tt * (c[0] - q[0]);
                    pv[v][1] = q[1] + tt * (c[1] - q[1]);
                }
                int i0 = 0, i1 = NR - 1, j0 = 0, j1 = NC - 1;
                if (proj) {
                    double amin = pv[0][0], amax = pv[0][0], bmin = pv[0][1], bmax = pv[0][1];
                    for (int v = 1; v < 3; ++v) {
                        if (pv[v][0] < amin) amin = pv[v][0];
                        if (pv[v][0] > amax) amax = pv[v][0];
                        if (pv[v][1] < bmin) bmin = pv[v][1];
                        if (pv[v][1] > bmax) bmax = pv[v][1];
                    }
                    double fa0 = floor(amin - mg), fa1 = ceil(amax + mg), fb0 = floor(bmin - mg), fb1 = ceil(bmax + mg);
                    if (fa0 > i0) i0 = fa0 > (double)NR ? NR : (int)fa0;
                    if (fa1 < i1) i1 = fa1 < -1.0 ? -1 : (int)fa1;
                    if (fb0 > j0) j0 = fb0 > (double)NC ? NC : (int)fb0;
                    if (fb1 < j1) j1 = fb1 < -1.0 ? -1 : (int)fb1;
                    /* vertices in light-plane units for the boundary distance */
                    for (int v = 0; v < 3; ++v) {
                        pv[v][0] *= sx;
                        pv[v][1] *= sy;
                    }
                } else {
                    ++fallback;
                }
                if (i0 > i1 || j0 > j1) continue;
                ++evald;
                for (int i = i0; i <= i1; ++i)
                    for (int j = j0; j <= j1; ++j) {
                        double mn = 1e300, dmin = 1e300;
                        for (int e = 0; e < planes; ++e) {
                            double val = A[e] * i + B[e] * j + C[e];
                            double v = val * inv[e];
                            if (v < mn) mn = v;
                            double dl = fabs(val) * pn[e];
                            if (dl < dmin) dmin = dl;
                        }
                        int b = i * NC + j;
                        double dist;
                        if (mn >= 0.0) {
                            if (!(mk[b >> 5] & (1u << (b & 31)))) ++nset;
                            mk[b >> 5] |= 1u << (b & 31);
                            dist = dmin;             /* inside: distance to the nearest edge */
                        } else if (!need_dist) {
                            continue;
                        } else if (proj) {
                            double px = i * sx, py = j * sy;
                            dist = o3_seg_dist(px, py, pv[0], pv[1]);
                            double d2 = o3_seg_dist(px, py, pv[1], pv[2]);
                            double d3 = o3_seg_dist(px, py, pv[2], pv[0]);
                            if (d2 < dist) dist = d2;
                            if (d3 < dist) dist = d3;
                        } else {
                            dist = 1e300;            /* outside an unbounded section: not attributed */
                        }
                        if (ed && dist < ed[b]) ed[b] = dist;
                    }
            }
        }
    }
    free(visit);
    }
    if (stats) {
        stats->candidates = cand;
        stats->evaluated = evald;
        stats->fallback = fallback;
        stats->skipped_blocks = skipped_blocks;
        stats->triangles = nt;
    }
    free(fv); free(tb); free(key); free(order); free(bb);
    free(recs);
}
