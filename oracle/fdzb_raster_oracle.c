/*
 * fdzb_raster_oracle.c -- CPU oracle of the G-buffer rasteriser (fdzb_raster_*).
 *
 * TEST INFRASTRUCTURE ONLY (see fdzb_oracle.h).  Build: oracle/Makefile, flags
 * -O2 -ffp-contract=off -fno-fast-math: every float expression below is one IEEE
 * binary32 operation per operator, in the written order, which the CUDA kernels
 * reproduce with __f*_rn intrinsics.
 *
 * What it restates: the app's G-buffer pass (4DZB/Render/Render.cpp:390-431,
 * DrawModel :267-340) with the gatherData shaders
 * (4DZB/Resources/shader/gatherData.shv/.shf): per vertex worldPos = M*(P,1),
 * worldN = M*(N,0), clip = VP*(worldPos,1); GL_TRIANGLES with the depth test
 * GL_LESS, depth cleared to 1 and colours to NaN; per fragment
 * G0 = (worldPos, Ks.r), G1 = (worldN, Ks.g), G2 = (Ka, Ks.b), G3 = (Kd,
 * shininess), worldPos and worldN interpolated perspective-correctly.  GL leaves
 * the exact rasterisation rules to the implementation; this rasteriser fixes
 * them (the CUDA kernels follow the same rules):
 *  - clipping: against the near plane z >= -w only (Sutherland-Hodgman in clip
 *    space, attributes interpolated linearly at t = d_a / (d_a - d_b)); the far
 *    plane is applied per fragment (0 <= depth <= 1), x and y by the viewport;
 *  - window coordinates x_w = x/w * (W/2) + W/2 (likewise y, row 0 at the
 *    bottom), depth z/w * 0.5 + 0.5, snapped to 1/16 pixel (round to nearest);
 *    a sub-triangle with a snapped coordinate beyond 2^26 pixels is dropped
 *    (counted);
 *  - coverage at pixel centres with exact 64-bit edge functions; a centre on an
 *    edge belongs to the triangle for which that edge, taken counter-clockwise,
 *    has dy < 0, or dy == 0 and dx > 0 -- exactly one of two triangles sharing
 *    the edge; zero-area triangles draw nothing; both windings are drawn;
 *  - depth: barycentric weights l_i = (float)E_i / (float)area, depth
 *    ((l0*z0 + l1*z1) + l2*z2); a fragment survives the GL_LESS test of the
 *    draw if no earlier fragment of the pixel has a smaller or equal depth,
 *    i.e. the winner is the least (depth, triangle order) pair -- the order of
 *    evaluation does not matter;
 *  - attributes: q_i = l_i * (1/w_i), a = ((q0*a0 + q1*a1) + q2*a2) /
 *    ((q0 + q1) + q2).
 */
#include "fdzb_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define RS_SUB 16                 /* subpixel steps per pixel */

typedef struct {
    float c[4];      /* clip x, y, z, w */
    float p[3], n[3];
} rs_vert;

typedef struct {
    long long X[3], Y[3];   /* snapped window coordinates, 1/16 px */
    float z[3], iw[3];
    float p[3][3], n[3][3];
    long long area;
    int tri, mat;
} rs_tri;

static void mat_vec4(const float m[16], const float v[4], float out[4])
{
    for (int r = 0; r < 4; ++r)
        out[r] = ((m[r] * v[0] + m[4 + r] * v[1]) + m[8 + r] * v[2]) + m[12 + r] * v[3];
}

static long long snap(float v)
{
    /* v * 16, rounded to nearest (ties to even, as __float2ll_rn) */
    float s = v * (float)RS_SUB;
    return llrintf(s);
}

/* vertex of the clipped polygon between a and b at t */
static rs_vert lerp_vert(const rs_vert *a, const rs_vert *b, float t)
{
    rs_vert o;
    for (int k = 0; k < 4; ++k) o.c[k] = a->c[k] + t * (b->c[k] - a->c[k]);
    for (int k = 0; k < 3; ++k) {
        o.p[k] = a->p[k] + t * (b->p[k] - a->p[k]);
        o.n[k] = a->n[k] + t * (b->n[k] - a->n[k]);
    }
    return o;
}

/* sub-triangle setup; returns 1 if it draws anything */
static int setup_sub(const rs_vert *v0, const rs_vert *v1, const rs_vert *v2, int W, int H, int tri, int mat,
                     rs_tri *o, int64_t *dropped)
{
    const rs_vert *v[3] = {v0, v1, v2};
    const float hw = 0.5f * (float)W, hh = 0.5f * (float)H;
    for (int i = 0; i < 3; ++i) {
        const float w = v[i]->c[3];
        if (!(w > 0.0f)) return 0;
        const float xn = v[i]->c[0] / w, yn = v[i]->c[1] / w, zn = v[i]->c[2] / w;
        const float xw = xn * hw + hw, yw = yn * hh + hh;
        if (!(fabsf(xw) < 67108864.0f && fabsf(yw) < 67108864.0f)) {
            ++*dropped;
            return 0;
        }
        o->X[i] = snap(xw);
        o->Y[i] = snap(yw);
        o->z[i] = zn * 0.5f + 0.5f;
        o->iw[i] = 1.0f / w;
        for (int k = 0; k < 3; ++k) {
            o->p[i][k] = v[i]->p[k];
            o->n[i][k] = v[i]->n[k];
        }
    }
    long long area = (o->X[1] - o->X[0]) * (o->Y[2] - o->Y[0]) - (o->Y[1] - o->Y[0]) * (o->X[2] - o->X[0]);
    if (area == 0) return 0;
    if (area < 0) {   /* make it counter-clockwise: swap vertices 1 and 2 */
        long long tx = o->X[1], ty = o->Y[1];
        o->X[1] = o->X[2]; o->Y[1] = o->Y[2]; o->X[2] = tx; o->Y[2] = ty;
        float tz = o->z[1]; o->z[1] = o->z[2]; o->z[2] = tz;
        float ti = o->iw[1]; o->iw[1] = o->iw[2]; o->iw[2] = ti;
        for (int k = 0; k < 3; ++k) {
            float a = o->p[1][k]; o->p[1][k] = o->p[2][k]; o->p[2][k] = a;
            float b = o->n[1][k]; o->n[1][k] = o->n[2][k]; o->n[2][k] = b;
        }
        area = -area;
    }
    o->area = area;
    o->tri = tri;
    o->mat = mat;
    return 1;
}

/* edge (a -> b), counter-clockwise: a centre exactly on it is inside when the
 * edge has dy < 0, or dy == 0 and dx > 0 */
static int edge_owns(long long ax, long long ay, long long bx, long long by)
{
    const long long dx = bx - ax, dy = by - ay;
    return dy < 0 || (dy == 0 && dx > 0);
}

int32_t orc_raster(const orc_raster_in *in, orc_raster_out *o)
{
    const int W = in->W, H = in->H;
    if (W <= 0 || H <= 0 || W > 16384 || H > 16384 || in->n_tri < 0) return -1;
    const size_t S = (size_t)W * H;
    const int sf = in->vtx_stride_floats;
    o->sub_tris = 0;
    o->dropped = 0;
    if (in->clear) {
        for (size_t i = 0; i < 4 * S; ++i) {
            o->g0[i] = NAN;
            o->g1[i] = NAN;
            if (o->g2) o->g2[i] = NAN;
            if (o->g3) o->g3[i] = NAN;
        }
        for (size_t i = 0; i < S; ++i) o->depth[i] = 1.0f;
    }
    /* winner per pixel: least (depth, order) of this draw */
    float *bz = (float *)malloc(sizeof(float) * S);
    long long *bid = (long long *)malloc(sizeof(long long) * S);
    rs_tri *subs = (rs_tri *)malloc(sizeof(rs_tri) * 2 * (size_t)(in->n_tri > 0 ? in->n_tri : 1));
    if (!bz || !bid || !subs) {
        free(bz); free(bid); free(subs);
        return -2;
    }
    for (size_t i = 0; i < S; ++i) {
        bz[i] = INFINITY;
        bid[i] = -1;
    }
    long long nsub = 0;
    for (int t = 0; t < in->n_tri; ++t) {
        rs_vert v[3];
        for (int i = 0; i < 3; ++i) {
            const float *src = in->vtx + (size_t)in->idx[3 * t + i] * sf;
            const float P[4] = {src[in->pos_offset], src[in->pos_offset + 1], src[in->pos_offset + 2], 1.0f};
            const float N[4] = {src[in->nrm_offset], src[in->nrm_offset + 1], src[in->nrm_offset + 2], 0.0f};
            float wp[4], wn[4];
            mat_vec4(in->model, P, wp);
            mat_vec4(in->model, N, wn);
            const float WP[4] = {wp[0], wp[1], wp[2], 1.0f};
            mat_vec4(in->view_proj, WP, v[i].c);
            for (int k = 0; k < 3; ++k) {
                v[i].p[k] = wp[k];
                v[i].n[k] = wn[k];
            }
        }
        const int mat = in->tri_material ? in->tri_material[t] : 0;
        /* near plane z >= -w: Sutherland-Hodgman */
        rs_vert poly[4];
        int np = 0;
        for (int i = 0; i < 3; ++i) {
            const rs_vert *a = &v[i], *b = &v[(i + 1) % 3];
            const float da = a->c[2] + a->c[3], db = b->c[2] + b->c[3];
            if (da >= 0.0f) poly[np++] = *a;
            if ((da >= 0.0f) != (db >= 0.0f)) poly[np++] = lerp_vert(a, b, da / (da - db));
        }
        if (np >= 3 && setup_sub(&poly[0], &poly[1], &poly[2], W, H, t, mat, &subs[nsub], &o->dropped)) ++nsub;
        if (np == 4 && setup_sub(&poly[0], &poly[2], &poly[3], W, H, t, mat, &subs[nsub], &o->dropped)) ++nsub;
    }
    o->sub_tris = nsub;
    for (long long si = 0; si < nsub; ++si) {
        const rs_tri *r = &subs[si];
        long long mnx = r->X[0], mxx = r->X[0], mny = r->Y[0], mxy = r->Y[0];
        for (int i = 1; i < 3; ++i) {
            if (r->X[i] < mnx) mnx = r->X[i];
            if (r->X[i] > mxx) mxx = r->X[i];
            if (r->Y[i] < mny) mny = r->Y[i];
            if (r->Y[i] > mxy) mxy = r->Y[i];
        }
        /* pixel centres x*16 + 8 inside [mnx, mxx] */
        long long x0 = (mnx - 8 + 15) >> 4, x1 = (mxx - 8) >> 4;
        long long y0 = (mny - 8 + 15) >> 4, y1 = (mxy - 8) >> 4;
        if (x0 < 0) x0 = 0;
        if (y0 < 0) y0 = 0;
        if (x1 > W - 1) x1 = W - 1;
        if (y1 > H - 1) y1 = H - 1;
        const int own0 = edge_owns(r->X[1], r->Y[1], r->X[2], r->Y[2]);
        const int own1 = edge_owns(r->X[2], r->Y[2], r->X[0], r->Y[0]);
        const int own2 = edge_owns(r->X[0], r->Y[0], r->X[1], r->Y[1]);
        const float fa = (float)r->area;
        for (long long y = y0; y <= y1; ++y)
            for (long long x = x0; x <= x1; ++x) {
                const long long px = x * 16 + 8, py = y * 16 + 8;
                const long long e0 = (r->X[2] - r->X[1]) * (py - r->Y[1]) - (r->Y[2] - r->Y[1]) * (px - r->X[1]);
                const long long e1 = (r->X[0] - r->X[2]) * (py - r->Y[2]) - (r->Y[0] - r->Y[2]) * (px - r->X[2]);
                const long long e2 = (r->X[1] - r->X[0]) * (py - r->Y[0]) - (r->Y[1] - r->Y[0]) * (px - r->X[0]);
                if (e0 < 0 || e1 < 0 || e2 < 0) continue;
                if ((e0 == 0 && !own0) || (e1 == 0 && !own1) || (e2 == 0 && !own2)) continue;
                const float l0 = (float)e0 / fa, l1 = (float)e1 / fa, l2 = (float)e2 / fa;
                const float z = (l0 * r->z[0] + l1 * r->z[1]) + l2 * r->z[2];
                if (!(z >= 0.0f && z <= 1.0f)) continue;
                const size_t p = (size_t)y * W + x;
                if (z < bz[p] || (z == bz[p] && si < bid[p])) {
                    bz[p] = z;
                    bid[p] = si;
                }
            }
    }
    for (size_t p = 0; p < S; ++p) {
        if (bid[p] < 0) continue;
        if (!(bz[p] < o->depth[p])) continue;   /* GL_LESS against earlier draws */
        const rs_tri *r = &subs[bid[p]];
        const long long x = (long long)(p % W), y = (long long)(p / W);
        const long long px = x * 16 + 8, py = y * 16 + 8;
        const long long e0 = (r->X[2] - r->X[1]) * (py - r->Y[1]) - (r->Y[2] - r->Y[1]) * (px - r->X[1]);
        const long long e1 = (r->X[0] - r->X[2]) * (py - r->Y[2]) - (r->Y[0] - r->Y[2]) * (px - r->X[2]);
        const long long e2 = (r->X[1] - r->X[0]) * (py - r->Y[0]) - (r->Y[1] - r->Y[0]) * (px - r->X[0]);
        const float fa = (float)r->area;
        const float l0 = (float)e0 / fa, l1 = (float)e1 / fa, l2 = (float)e2 / fa;
        const float q0 = l0 * r->iw[0], q1 = l1 * r->iw[1], q2 = l2 * r->iw[2];
        const float d = (q0 + q1) + q2;
        float P[3], N[3];
        for (int k = 0; k < 3; ++k) {
            P[k] = ((q0 * r->p[0][k] + q1 * r->p[1][k]) + q2 * r->p[2][k]) / d;
            N[k] = ((q0 * r->n[0][k] + q1 * r->n[1][k]) + q2 * r->n[2][k]) / d;
        }
        const float *m = in->materials + 10 * (size_t)r->mat;
        o->depth[p] = bz[p];
        float *g0 = o->g0 + 4 * p, *g1 = o->g1 + 4 * p;
        g0[0] = P[0]; g0[1] = P[1]; g0[2] = P[2]; g0[3] = m[6];
        g1[0] = N[0]; g1[1] = N[1]; g1[2] = N[2]; g1[3] = m[7];
        if (o->g2) {
            float *g2 = o->g2 + 4 * p;
            g2[0] = m[0]; g2[1] = m[1]; g2[2] = m[2]; g2[3] = m[8];
        }
        if (o->g3) {
            float *g3 = o->g3 + 4 * p;
            g3[0] = m[3]; g3[1] = m[4]; g3[2] = m[5]; g3[3] = m[9];
        }
    }
    free(bz);
    free(bid);
    free(subs);
    return 0;
}
