// fdzb_raster.cu -- G-buffer rasteriser: the view samples' producer.
//
// Replaces the app's GL G-buffer pass (4DZB/Render/Render.cpp:390-431 and
// DrawModel :267-340 with the gatherData shaders, 4DZB/Resources/shader/
// gatherData.shv/.shf) so that meshes feed the shadow pipeline without a
// graphics stack.  Per vertex worldPos = model*(P,1), worldN = model*(N,0),
// clip = view_proj*(worldPos,1); per pixel the nearest fragment (GL_LESS,
// earlier triangle wins ties) writes g0 = (worldPos, Ks.r), g1 = (worldN,
// Ks.g), g2 = (Ka, Ks.b), g3 = (Kd, shininess), worldPos and worldN
// interpolated perspective-correctly.  The rules GL leaves open are fixed (and
// restated by the oracle, oracle/fdzb_raster_oracle.c): near-plane clipping in
// clip space, window coordinates snapped to 1/16 pixel, coverage at pixel
// centres by exact 64-bit edge functions with an ownership rule for centres on
// an edge, depth 0..1 per fragment.  Every float operation is an _rn
// intrinsic, so the result is the oracle's bit for bit.
//
// B200 layout: one thread per triangle sets up at most two sub-triangles (the
// near-plane clip of a triangle is a triangle or a quad) into 144-byte records
// at slots 2t and 2t+1, and counts the 16 x 16 pixel tiles their pixel boxes
// touch; an exclusive scan over tiles sizes the tile lists; a scatter fills
// them; one 256-thread block per non-empty tile stages its list 32 records at
// a time in shared memory and keeps, per pixel (one thread each), the least
// (depth, slot) -- the GL_LESS winner whatever the order of evaluation -- and
// finally resolves the winner's attributes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "../../include/fdzb.h"
#include "fdzb_device.cuh"
#include "fdzb_internal.h"

namespace fdzb {
namespace {

constexpr int kTile = 16;              // pixels per tile side
constexpr int kRecF4 = 9;              // float4s per sub-triangle record
constexpr int kChunk = 32;             // records staged per round
constexpr float kMaxWindow = 67108864.0f;   // 2^26 pixels

struct RasterCounters {
    unsigned long long subTris, dropped, pairs, badIdx, badMat;
};

struct RVert {
    float c[4];
    float p[3], n[3];
};

__device__ __forceinline__ void mat_vec4(const float *m, const float v[4], float out[4])
{
#pragma unroll
    for (int r = 0; r < 4; ++r)
        out[r] = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[r], v[0]), __fmul_rn(m[4 + r], v[1])),
                                     __fmul_rn(m[8 + r], v[2])),
                           __fmul_rn(m[12 + r], v[3]));
}

__device__ __forceinline__ float lerp_rn(float a, float b, float t) { return __fadd_rn(a, __fmul_rn(t, __fsub_rn(b, a))); }

__device__ __forceinline__ RVert lerp_vert(const RVert &a, const RVert &b, float t)
{
    RVert o;
#pragma unroll
    for (int k = 0; k < 4; ++k) o.c[k] = lerp_rn(a.c[k], b.c[k], t);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        o.p[k] = lerp_rn(a.p[k], b.p[k], t);
        o.n[k] = lerp_rn(a.n[k], b.n[k], t);
    }
    return o;
}

struct SubTri {
    int X[3], Y[3];
    long long area;
    float z[3], iw[3];
    float p[3][3], n[3][3];
};

// Window setup of one sub-triangle; returns 1 if it can draw (non-zero area,
// every vertex in front and inside the 2^26-pixel window range), 2 if dropped.
__device__ int setup_sub(const RVert &a, const RVert &b, const RVert &c, int W, int H, SubTri &o)
{
    const RVert *v[3] = {&a, &b, &c};
    const float hw = __fmul_rn(0.5f, (float)W), hh = __fmul_rn(0.5f, (float)H);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float w = v[i]->c[3];
        if (!(w > 0.0f)) return 0;
        const float xn = __fdiv_rn(v[i]->c[0], w), yn = __fdiv_rn(v[i]->c[1], w), zn = __fdiv_rn(v[i]->c[2], w);
        const float xw = __fadd_rn(__fmul_rn(xn, hw), hw), yw = __fadd_rn(__fmul_rn(yn, hh), hh);
        if (!(fabsf(xw) < kMaxWindow && fabsf(yw) < kMaxWindow)) return 2;
        o.X[i] = (int)__float2ll_rn(__fmul_rn(xw, 16.0f));
        o.Y[i] = (int)__float2ll_rn(__fmul_rn(yw, 16.0f));
        o.z[i] = __fadd_rn(__fmul_rn(zn, 0.5f), 0.5f);
        o.iw[i] = __fdiv_rn(1.0f, w);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            o.p[i][k] = v[i]->p[k];
            o.n[i][k] = v[i]->n[k];
        }
    }
    long long area = (long long)(o.X[1] - o.X[0]) * (long long)(o.Y[2] - o.Y[0]) -
                     (long long)(o.Y[1] - o.Y[0]) * (long long)(o.X[2] - o.X[0]);
    if (area == 0) return 0;
    if (area < 0) {   // counter-clockwise: swap vertices 1 and 2
        int t = o.X[1]; o.X[1] = o.X[2]; o.X[2] = t;
        t = o.Y[1]; o.Y[1] = o.Y[2]; o.Y[2] = t;
        float f = o.z[1]; o.z[1] = o.z[2]; o.z[2] = f;
        f = o.iw[1]; o.iw[1] = o.iw[2]; o.iw[2] = f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            f = o.p[1][k]; o.p[1][k] = o.p[2][k]; o.p[2][k] = f;
            f = o.n[1][k]; o.n[1][k] = o.n[2][k]; o.n[2][k] = f;
        }
        area = -area;
    }
    o.area = area;
    return 1;
}

// Pixel-centre box of a sub-triangle, clamped to the viewport (x0 > x1: none).
__device__ __forceinline__ void pixel_box(const int *X, const int *Y, int W, int H, int &x0, int &x1, int &y0,
                                          int &y1)
{
    const int mnx = min(X[0], min(X[1], X[2])), mxx = max(X[0], max(X[1], X[2]));
    const int mny = min(Y[0], min(Y[1], Y[2])), mxy = max(Y[0], max(Y[1], Y[2]));
    // centres x*16 + 8 inside [mnx, mxx]
    x0 = max((mnx - 8 + 15) >> 4, 0);
    x1 = min((mxx - 8) >> 4, W - 1);
    y0 = max((mny - 8 + 15) >> 4, 0);
    y1 = min((mxy - 8) >> 4, H - 1);
}

__device__ __forceinline__ void store_record(float4 *rec, const SubTri &s, int mat, int valid)
{
    rec[0] = make_float4(__int_as_float(s.X[0]), __int_as_float(s.Y[0]), __int_as_float(s.X[1]),
                         __int_as_float(s.Y[1]));
    rec[1] = make_float4(__int_as_float(s.X[2]), __int_as_float(s.Y[2]), __int_as_float((int)(s.area & 0xffffffffll)),
                         __int_as_float((int)(s.area >> 32)));
    rec[2] = make_float4(s.z[0], s.z[1], s.z[2], s.iw[0]);
    rec[3] = make_float4(s.iw[1], s.iw[2], __int_as_float(mat), __int_as_float(valid));
    rec[4] = make_float4(s.p[0][0], s.p[0][1], s.p[0][2], s.p[1][0]);
    rec[5] = make_float4(s.p[1][1], s.p[1][2], s.p[2][0], s.p[2][1]);
    rec[6] = make_float4(s.p[2][2], s.n[0][0], s.n[0][1], s.n[0][2]);
    rec[7] = make_float4(s.n[1][0], s.n[1][1], s.n[1][2], s.n[2][0]);
    rec[8] = make_float4(s.n[2][1], s.n[2][2], 0.0f, 0.0f);
}

__device__ __forceinline__ void count_tiles(const SubTri &s, int W, int H, int tilesX, int *tileCount,
                                            unsigned long long &pairs)
{
    int x0, x1, y0, y1;
    pixel_box(s.X, s.Y, W, H, x0, x1, y0, y1);
    if (x0 > x1 || y0 > y1) return;
    for (int ty = y0 / kTile; ty <= y1 / kTile; ++ty)
        for (int tx = x0 / kTile; tx <= x1 / kTile; ++tx) {
            atomicAdd(&tileCount[ty * tilesX + tx], 1);
            ++pairs;
        }
}

__global__ void k_rs_clear(int S, float4 *g0, float4 *g1, float4 *g2, float4 *g3, float *depth)
{
    const float nan = __int_as_float(0x7fc00000);
    const float4 q = make_float4(nan, nan, nan, nan);
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < S; p += gridDim.x * blockDim.x) {
        g0[p] = q;
        g1[p] = q;
        if (g2) g2[p] = q;
        if (g3) g3[p] = q;
        depth[p] = 1.0f;
    }
}

__global__ void __launch_bounds__(128) k_rs_setup(const float *__restrict__ vtx, int V, int strideF, int posOff,
                                                  int nrmOff, const uint32_t *__restrict__ idx, int T,
                                                  const int32_t *__restrict__ triMat, int nMat, const float *model,
                                                  const float *viewProj, int W, int H, int tilesX,
                                                  float4 *__restrict__ recs, int *__restrict__ tileCount,
                                                  RasterCounters *ctr)
{
    __shared__ float sM[16], sVP[16];
    if (threadIdx.x < 16) {
        sM[threadIdx.x] = model[threadIdx.x];
        sVP[threadIdx.x] = viewProj[threadIdx.x];
    }
    __syncthreads();
    unsigned long long nsub = 0, ndrop = 0, npairs = 0, nbadI = 0, nbadM = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        float4 *r0 = recs + (size_t)kRecF4 * (2 * (size_t)t);
        float4 *r1 = r0 + kRecF4;
        r0[3].w = __int_as_float(0);
        r1[3].w = __int_as_float(0);
        RVert v[3];
        bool ok = true;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const uint32_t id = idx[3 * (size_t)t + i];
            if (id >= (uint32_t)V) {
                ok = false;
                break;
            }
            const float *src = vtx + (size_t)id * strideF;
            const float P[4] = {src[posOff], src[posOff + 1], src[posOff + 2], 1.0f};
            const float N[4] = {src[nrmOff], src[nrmOff + 1], src[nrmOff + 2], 0.0f};
            float wp[4], wn[4];
            mat_vec4(sM, P, wp);
            mat_vec4(sM, N, wn);
            const float WP[4] = {wp[0], wp[1], wp[2], 1.0f};
            mat_vec4(sVP, WP, v[i].c);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                v[i].p[k] = wp[k];
                v[i].n[k] = wn[k];
            }
        }
        if (!ok) {
            ++nbadI;
            continue;
        }
        int mat = triMat ? triMat[t] : 0;
        if (mat < 0 || mat >= nMat) {
            ++nbadM;
            mat = 0;
        }
        // near plane z >= -w (Sutherland-Hodgman)
        RVert poly[4];
        int np = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const RVert &a = v[i], &b = v[(i + 1) % 3];
            const float da = __fadd_rn(a.c[2], a.c[3]), db = __fadd_rn(b.c[2], b.c[3]);
            if (da >= 0.0f) poly[np++] = a;
            if ((da >= 0.0f) != (db >= 0.0f)) poly[np++] = lerp_vert(a, b, __fdiv_rn(da, __fsub_rn(da, db)));
        }
        SubTri s;
        if (np >= 3) {
            const int rc = setup_sub(poly[0], poly[1], poly[2], W, H, s);
            if (rc == 2) ++ndrop;
            if (rc == 1) {
                store_record(r0, s, mat, 1);
                ++nsub;
                count_tiles(s, W, H, tilesX, tileCount, npairs);
            }
        }
        if (np == 4) {
            const int rc = setup_sub(poly[0], poly[2], poly[3], W, H, s);
            if (rc == 2) ++ndrop;
            if (rc == 1) {
                store_record(r1, s, mat, 1);
                ++nsub;
                count_tiles(s, W, H, tilesX, tileCount, npairs);
            }
        }
    }
    if (nsub) atomicAdd(&ctr->subTris, nsub);
    if (ndrop) atomicAdd(&ctr->dropped, ndrop);
    if (npairs) atomicAdd(&ctr->pairs, npairs);
    if (nbadI) atomicAdd(&ctr->badIdx, nbadI);
    if (nbadM) atomicAdd(&ctr->badMat, nbadM);
}

// Exclusive scan of the tile counts (one block).
__global__ void __launch_bounds__(1024) k_rs_scan(const int *__restrict__ cnt, int *__restrict__ start, int n)
{
    __shared__ long long part[1024];
    const int per = (n + 1023) / 1024;
    const int lo = min(n, threadIdx.x * per), hi = min(n, lo + per);
    long long s = 0;
    for (int i = lo; i < hi; ++i) s += cnt[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const long long v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    long long run = threadIdx.x ? part[threadIdx.x - 1] : 0;
    for (int i = lo; i < hi; ++i) {
        start[i] = (int)run;
        run += cnt[i];
    }
}

__global__ void k_rs_scatter(const float4 *__restrict__ recs, int slots, int W, int H, int tilesX,
                             const int *__restrict__ tileStart, int *__restrict__ tileFill, int *__restrict__ pairs,
                             long long capacity)
{
    for (int sl = blockIdx.x * blockDim.x + threadIdx.x; sl < slots; sl += gridDim.x * blockDim.x) {
        const float4 *r = recs + (size_t)kRecF4 * sl;
        if (!__float_as_int(r[3].w)) continue;
        const float4 a = r[0], b = r[1];
        const int X[3] = {__float_as_int(a.x), __float_as_int(a.z), __float_as_int(b.x)};
        const int Y[3] = {__float_as_int(a.y), __float_as_int(a.w), __float_as_int(b.y)};
        int x0, x1, y0, y1;
        pixel_box(X, Y, W, H, x0, x1, y0, y1);
        if (x0 > x1 || y0 > y1) continue;
        for (int ty = y0 / kTile; ty <= y1 / kTile; ++ty)
            for (int tx = x0 / kTile; tx <= x1 / kTile; ++tx) {
                const int tile = ty * tilesX + tx;
                const long long pos = (long long)tileStart[tile] + atomicAdd(&tileFill[tile], 1);
                if (pos < capacity) pairs[pos] = sl;
            }
    }
}

// edge (a -> b), counter-clockwise: a centre exactly on it is inside when the
// edge has dy < 0, or dy == 0 and dx > 0
__device__ __forceinline__ bool edge_owns(int ax, int ay, int bx, int by)
{
    const int dx = bx - ax, dy = by - ay;
    return dy < 0 || (dy == 0 && dx > 0);
}

__device__ __forceinline__ long long edge_fn(int ax, int ay, int bx, int by, long long px, long long py)
{
    return (long long)(bx - ax) * (py - ay) - (long long)(by - ay) * (px - ax);
}

__global__ void __launch_bounds__(kTile * kTile) k_rs_tiles(const float4 *__restrict__ recs,
                                                            const int *__restrict__ tileCount,
                                                            const int *__restrict__ tileStart,
                                                            const int *__restrict__ pairs, long long capacity,
                                                            int W, int H, int tilesX, int clear,
                                                            const float *__restrict__ mats, float4 *g0, float4 *g1,
                                                            float4 *g2, float4 *g3, float *depth)
{
    __shared__ float4 s_rec[kChunk][4];   // geometry and depth part of each record
    __shared__ int s_slot[kChunk];
    const int tile = blockIdx.x;
    const int n = tileCount[tile];
    if (n == 0) return;
    const int base = tileStart[tile];
    const int px = (tile % tilesX) * kTile + (threadIdx.x & (kTile - 1));
    const int py = (tile / tilesX) * kTile + (threadIdx.x / kTile);
    const bool inside = px < W && py < H;
    const long long cx = (long long)px * 16 + 8, cy = (long long)py * 16 + 8;
    float bz = __int_as_float(0x7f800000);   // +inf
    int bslot = 0x7fffffff;
    for (int c0 = 0; c0 < n; c0 += kChunk) {
        const int m = min(kChunk, n - c0);
        __syncthreads();
        if (threadIdx.x < m * 4) {
            const int k = threadIdx.x >> 2, part = threadIdx.x & 3;
            const long long pi = (long long)base + c0 + k;
            const int sl = pi < capacity ? pairs[pi] : 0;
            s_rec[k][part] = recs[(size_t)kRecF4 * sl + part];
            if (part == 0) s_slot[k] = sl;
        }
        __syncthreads();
        if (!inside) continue;
        for (int k = 0; k < m; ++k) {
            const float4 a = s_rec[k][0], b = s_rec[k][1];
            const int X0 = __float_as_int(a.x), Y0 = __float_as_int(a.y), X1 = __float_as_int(a.z),
                      Y1 = __float_as_int(a.w), X2 = __float_as_int(b.x), Y2 = __float_as_int(b.y);
            const long long e0 = edge_fn(X1, Y1, X2, Y2, cx, cy);
            const long long e1 = edge_fn(X2, Y2, X0, Y0, cx, cy);
            const long long e2 = edge_fn(X0, Y0, X1, Y1, cx, cy);
            if (e0 < 0 || e1 < 0 || e2 < 0) continue;
            if ((e0 == 0 && !edge_owns(X1, Y1, X2, Y2)) || (e1 == 0 && !edge_owns(X2, Y2, X0, Y0)) ||
                (e2 == 0 && !edge_owns(X0, Y0, X1, Y1)))
                continue;
            const long long area = (long long)(unsigned)__float_as_int(b.z) | ((long long)__float_as_int(b.w) << 32);
            const float fa = __ll2float_rn(area);
            const float l0 = __fdiv_rn(__ll2float_rn(e0), fa), l1 = __fdiv_rn(__ll2float_rn(e1), fa),
                        l2 = __fdiv_rn(__ll2float_rn(e2), fa);
            const float4 zz = s_rec[k][2];
            const float z = __fadd_rn(__fadd_rn(__fmul_rn(l0, zz.x), __fmul_rn(l1, zz.y)), __fmul_rn(l2, zz.z));
            if (!(z >= 0.0f && z <= 1.0f)) continue;
            const int sl = s_slot[k];
            if (z < bz || (z == bz && sl < bslot)) {
                bz = z;
                bslot = sl;
            }
        }
    }
    if (!inside || bslot == 0x7fffffff) return;
    const size_t p = (size_t)py * W + px;
    if (!clear && !(bz < depth[p])) return;   // GL_LESS against earlier draws
    const float4 *r = recs + (size_t)kRecF4 * bslot;
    const float4 a = r[0], b = r[1], r2 = r[2], r3 = r[3], r4 = r[4], r5 = r[5], r6 = r[6], r7 = r[7], r8 = r[8];
    const int X0 = __float_as_int(a.x), Y0 = __float_as_int(a.y), X1 = __float_as_int(a.z), Y1 = __float_as_int(a.w),
              X2 = __float_as_int(b.x), Y2 = __float_as_int(b.y);
    const long long e0 = edge_fn(X1, Y1, X2, Y2, cx, cy);
    const long long e1 = edge_fn(X2, Y2, X0, Y0, cx, cy);
    const long long e2 = edge_fn(X0, Y0, X1, Y1, cx, cy);
    const long long area = (long long)(unsigned)__float_as_int(b.z) | ((long long)__float_as_int(b.w) << 32);
    const float fa = __ll2float_rn(area);
    const float l0 = __fdiv_rn(__ll2float_rn(e0), fa), l1 = __fdiv_rn(__ll2float_rn(e1), fa),
                l2 = __fdiv_rn(__ll2float_rn(e2), fa);
    const float q0 = __fmul_rn(l0, r2.w), q1 = __fmul_rn(l1, r3.x), q2 = __fmul_rn(l2, r3.y);
    const float d = __fadd_rn(__fadd_rn(q0, q1), q2);
    const float P0[3] = {r4.x, r4.y, r4.z}, P1[3] = {r4.w, r5.x, r5.y}, P2[3] = {r5.z, r5.w, r6.x};
    const float N0[3] = {r6.y, r6.z, r6.w}, N1[3] = {r7.x, r7.y, r7.z}, N2[3] = {r7.w, r8.x, r8.y};
    float P[3], N[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        P[k] = __fdiv_rn(__fadd_rn(__fadd_rn(__fmul_rn(q0, P0[k]), __fmul_rn(q1, P1[k])), __fmul_rn(q2, P2[k])), d);
        N[k] = __fdiv_rn(__fadd_rn(__fadd_rn(__fmul_rn(q0, N0[k]), __fmul_rn(q1, N1[k])), __fmul_rn(q2, N2[k])), d);
    }
    const float *mt = mats + 10 * (size_t)__float_as_int(r3.z);
    depth[p] = bz;
    g0[p] = make_float4(P[0], P[1], P[2], mt[6]);
    g1[p] = make_float4(N[0], N[1], N[2], mt[7]);
    if (g2) g2[p] = make_float4(mt[0], mt[1], mt[2], mt[8]);
    if (g3) g3[p] = make_float4(mt[3], mt[4], mt[5], mt[9]);
}

}  // namespace
}  // namespace fdzb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
static_assert(sizeof(fdzb_raster_desc) == 240, "fdzb_raster_desc layout");
static_assert(sizeof(fdzb_raster_stats) == 64, "fdzb_raster_stats layout");

struct fdzb_raster {
    int device = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float4 *recs = nullptr;
    size_t recSlots = 0;
    int *tileCount = nullptr, *tileStart = nullptr, *tileFill = nullptr;
    size_t tileCap = 0;
    int *pairs = nullptr;
    long long pairCap = 0;
    float *depthScratch = nullptr;
    size_t depthCap = 0;
    float *dMats = nullptr;   // model and view_proj
    fdzb::RasterCounters *ctr = nullptr, *hCtr = nullptr;
    fdzb_raster_stats stats{};
    bool pending = false;
};

namespace {

int rfail(int code, const std::string &msg) { return fdzb::set_error(code, "fdzb_raster: " + msg); }

#define RS_CUDA(call)                                                                         \
    do {                                                                                      \
        cudaError_t _e = (call);                                                              \
        if (_e != cudaSuccess) return rfail(FDZB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
    } while (0)

int grow(void **p, size_t &cap, size_t need, size_t elem)
{
    if (need <= cap) return FDZB_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    cap = 0;
    size_t n = need + need / 4 + 64;
    if (cudaMalloc(p, n * elem) != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return rfail(FDZB_ERR_NO_MEMORY, "device allocation failed");
    }
    cap = n;
    return FDZB_OK;
}

int finish(fdzb_raster *r)
{
    if (!r->pending) return FDZB_OK;
    RS_CUDA(cudaEventSynchronize(r->e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r->e0, r->e1);
    r->stats.ms = ms;
    r->pending = false;
    return FDZB_OK;
}

}  // namespace

extern "C" {

int fdzb_raster_create(fdzb_raster **out, int device)
{
    if (!out) return rfail(FDZB_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    int dev = device;
    if (dev < 0) RS_CUDA(cudaGetDevice(&dev));
    RS_CUDA(cudaSetDevice(dev));
    fdzb_raster *r = new fdzb_raster();
    r->device = dev;
    if (cudaStreamCreateWithFlags(&r->own, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&r->e0) != cudaSuccess || cudaEventCreate(&r->e1) != cudaSuccess ||
        cudaMalloc(&r->dMats, 32 * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&r->ctr, sizeof(fdzb::RasterCounters)) != cudaSuccess ||
        cudaMallocHost(&r->hCtr, sizeof(fdzb::RasterCounters)) != cudaSuccess) {
        cudaGetLastError();
        fdzb_raster_destroy(r);
        return rfail(FDZB_ERR_CUDA, "could not create the rasteriser's stream, events or buffers");
    }
    r->stream = r->own;
    *out = r;
    return FDZB_OK;
}

int fdzb_raster_destroy(fdzb_raster *r)
{
    if (!r) return FDZB_OK;
    cudaSetDevice(r->device);
    if (r->stream) cudaStreamSynchronize(r->stream);
    cudaFree(r->recs);
    cudaFree(r->tileCount);
    cudaFree(r->tileStart);
    cudaFree(r->tileFill);
    cudaFree(r->pairs);
    cudaFree(r->depthScratch);
    cudaFree(r->dMats);
    cudaFree(r->ctr);
    if (r->hCtr) cudaFreeHost(r->hCtr);
    if (r->e0) cudaEventDestroy(r->e0);
    if (r->e1) cudaEventDestroy(r->e1);
    if (r->own) cudaStreamDestroy(r->own);
    delete r;
    return FDZB_OK;
}

int fdzb_raster_set_stream(fdzb_raster *r, void *stream)
{
    if (!r) return rfail(FDZB_ERR_INVALID_ARG, "handle is NULL");
    if (int rc = finish(r)) return rc;
    r->stream = stream ? (cudaStream_t)stream : r->own;
    return FDZB_OK;
}

int fdzb_raster_sync(fdzb_raster *r)
{
    if (!r) return rfail(FDZB_ERR_INVALID_ARG, "handle is NULL");
    cudaSetDevice(r->device);
    return finish(r);
}

int fdzb_raster_get_stats(fdzb_raster *r, fdzb_raster_stats *st)
{
    if (!r || !st) return rfail(FDZB_ERR_INVALID_ARG, "NULL argument");
    if (int rc = fdzb_raster_sync(r)) return rc;
    *st = r->stats;
    return FDZB_OK;
}

int fdzb_raster_draw(fdzb_raster *r, const fdzb_raster_desc *d)
{
    using namespace fdzb;
    if (!r || !d) return rfail(FDZB_ERR_INVALID_ARG, "NULL argument");
    if (d->W < 1 || d->H < 1 || d->W > 16384 || d->H > 16384) return rfail(FDZB_ERR_INVALID_ARG, "W, H must be in 1..16384");
    if (d->n_tri < 0 || d->n_vtx < 0) return rfail(FDZB_ERR_INVALID_ARG, "negative count");
    if (d->n_tri > (1 << 29)) return rfail(FDZB_ERR_INVALID_ARG, "too many triangles (max 2^29)");
    if (d->n_tri > 0 && (!d->d_vtx || !d->d_idx)) return rfail(FDZB_ERR_INVALID_ARG, "NULL vertex or index buffer");
    if (d->vtx_stride_bytes < 12 || d->vtx_stride_bytes % 4) return rfail(FDZB_ERR_INVALID_ARG, "vertex stride must be >= 12, a multiple of 4");
    const int strideF = d->vtx_stride_bytes / 4;
    if (d->pos_offset < 0 || d->nrm_offset < 0 || d->pos_offset + 3 > strideF || d->nrm_offset + 3 > strideF)
        return rfail(FDZB_ERR_INVALID_ARG, "position / normal offsets outside the vertex");
    if (!d->d_materials || d->n_materials < 1) return rfail(FDZB_ERR_INVALID_ARG, "at least one material is required");
    if (!d->d_g0 || !d->d_g1) return rfail(FDZB_ERR_INVALID_ARG, "g0 and g1 are required");
    for (const void *p : {(const void *)d->d_g0, (const void *)d->d_g1, (const void *)d->d_g2, (const void *)d->d_g3})
        if ((uintptr_t)p & 15) return rfail(FDZB_ERR_INVALID_ARG, "G-buffer targets must be 16-byte aligned float4 arrays");
    if (!d->clear && !d->d_depth) return rfail(FDZB_ERR_INVALID_ARG, "drawing without clear needs the earlier draw's depth buffer");
    cudaSetDevice(r->device);
    if (int rc = finish(r)) return rc;

    const int W = d->W, H = d->H;
    const size_t S = (size_t)W * H;
    const int tilesX = (W + 15) / 16, tilesY = (H + 15) / 16;
    const size_t nTiles = (size_t)tilesX * tilesY;
    float *depth = d->d_depth;
    if (!depth) {
        if (int rc = grow((void **)&r->depthScratch, r->depthCap, S, sizeof(float))) return rc;
        depth = r->depthScratch;
    }
    if (int rc = grow((void **)&r->recs, r->recSlots, 2 * (size_t)std::max(d->n_tri, 1), kRecF4 * sizeof(float4))) return rc;
    if (nTiles > r->tileCap) {
        // the three per-tile arrays share one capacity
        cudaFree(r->tileCount);
        cudaFree(r->tileStart);
        cudaFree(r->tileFill);
        r->tileCount = r->tileStart = r->tileFill = nullptr;
        r->tileCap = 0;
        const size_t cap = nTiles + nTiles / 4 + 64;
        if (cudaMalloc(&r->tileCount, cap * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&r->tileStart, cap * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&r->tileFill, cap * sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            return rfail(FDZB_ERR_NO_MEMORY, "device allocation failed");
        }
        r->tileCap = cap;
    }
    cudaStream_t s = r->stream;
    int sm = 148;
    cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, r->device);
    float mats[32];
    std::memcpy(mats, d->model, sizeof(d->model));
    std::memcpy(mats + 16, d->view_proj, sizeof(d->view_proj));
    RS_CUDA(cudaEventRecord(r->e0, s));
    RS_CUDA(cudaMemcpyAsync(r->dMats, mats, sizeof(mats), cudaMemcpyHostToDevice, s));
    RS_CUDA(cudaMemsetAsync(r->ctr, 0, sizeof(RasterCounters), s));
    RS_CUDA(cudaMemsetAsync(r->tileCount, 0, nTiles * sizeof(int), s));
    RS_CUDA(cudaMemsetAsync(r->tileFill, 0, nTiles * sizeof(int), s));
    if (d->clear) {
        const int g = (int)std::min<size_t>((S + 255) / 256, (size_t)sm * 8);
        k_rs_clear<<<g, 256, 0, s>>>((int)S, (float4 *)d->d_g0, (float4 *)d->d_g1, (float4 *)d->d_g2,
                                     (float4 *)d->d_g3, depth);
    }
    if (d->n_tri > 0) {
        const int g = (int)std::min<long long>((d->n_tri + 127) / 128, (long long)sm * 16);
        k_rs_setup<<<g, 128, 0, s>>>(d->d_vtx, d->n_vtx, strideF, d->pos_offset, d->nrm_offset, d->d_idx, d->n_tri,
                                     d->d_tri_material, d->n_materials, r->dMats, r->dMats + 16, W, H, tilesX,
                                     r->recs, r->tileCount, r->ctr);
        k_rs_scan<<<1, 1024, 0, s>>>(r->tileCount, r->tileStart, (int)nTiles);
    }
    RS_CUDA(cudaGetLastError());
    RS_CUDA(cudaMemcpyAsync(r->hCtr, r->ctr, sizeof(RasterCounters), cudaMemcpyDeviceToHost, s));
    RS_CUDA(cudaStreamSynchronize(s));
    const RasterCounters c = *r->hCtr;
    r->stats = fdzb_raster_stats{};
    r->stats.triangles = d->n_tri;
    r->stats.sub_triangles = (int64_t)c.subTris;
    r->stats.dropped = (int64_t)c.dropped;
    r->stats.tile_pairs = (int64_t)c.pairs;
    r->stats.bad_indices = (int64_t)c.badIdx;
    r->stats.bad_materials = (int64_t)c.badMat;
    r->stats.tiles_x = tilesX;
    r->stats.tiles_y = tilesY;
    if (c.pairs > (unsigned long long)0x7fffffff) return rfail(FDZB_ERR_CAPACITY, "more than 2^31 tile pairs in one draw");
    if (d->n_tri > 0 && c.pairs > 0) {
        size_t pc = (size_t)r->pairCap;
        if (int rc = grow((void **)&r->pairs, pc, (size_t)c.pairs, sizeof(int))) return rc;
        r->pairCap = (long long)pc;
        const int slots = 2 * d->n_tri;
        const int g = (int)std::min<long long>((slots + 255) / 256, (long long)sm * 16);
        k_rs_scatter<<<g, 256, 0, s>>>(r->recs, slots, W, H, tilesX, r->tileStart, r->tileFill, r->pairs, r->pairCap);
        k_rs_tiles<<<(unsigned)nTiles, 256, 0, s>>>(r->recs, r->tileCount, r->tileStart, r->pairs, r->pairCap, W, H,
                                                    tilesX, d->clear, d->d_materials, (float4 *)d->d_g0,
                                                    (float4 *)d->d_g1, (float4 *)d->d_g2, (float4 *)d->d_g3, depth);
        RS_CUDA(cudaGetLastError());
    }
    RS_CUDA(cudaEventRecord(r->e1, s));
    r->pending = true;
    return FDZB_OK;
}

}  // extern "C"
