// fdzb_occlusion.cuh -- per-bin occlusion and popcount shading (stages c + d).
//
// Reference: shadowCal_per_sample_kernel (K/Step5_2_shadowCalPerSample.inl:37-231),
// one thread per sample walking its bin's triangle list through texture fetches.
//
// Here a warp owns a work item: up to kItemSamples samples of one bin.  The bin's
// triangle records are staged into shared memory kOccChunk at a time, together
// with the per-triangle values every pair test of the reference recomputes
// (the face normal cross(v1-v0, v2-v1) and the edge vectors v0-v1, v1-v2,
// v2-v0, each the same IEEE operation sequence).  Every lane tests its own
// sample against the staged triangles.  A lane whose sample is done (all light
// rows full -- the reference's early-out -- or every triangle seen) writes its
// result and, at the next chunk boundary, takes the next sample of the item;
// the warp streams the triangle list cyclically and each lane stops after
// exactly one full cycle.  The final mask is the OR over the tested triangles,
// so it is independent of the order and of where in the cycle a lane starts.
#pragma once
#include <type_traits>
#include "fdzb_device.cuh"

namespace fdzb {

#ifndef FDZB_OCC_REFILL
#define FDZB_OCC_REFILL 0
#endif
#ifndef FDZB_OCC_MINBLOCKS
#define FDZB_OCC_MINBLOCKS 7
#endif

#ifndef FDZB_OCC_ITEM
#define FDZB_OCC_ITEM 32
#endif
#ifndef FDZB_OCC_CHUNK
#define FDZB_OCC_CHUNK 32
#endif
#ifndef FDZB_OCC_VOTE
#define FDZB_OCC_VOTE 1
#endif


constexpr int kOccWarps = 4;
constexpr int kOccThreads = kOccWarps * 32;
constexpr int kOccChunk = FDZB_OCC_CHUNK;
static_assert(kOccChunk >= 1 && kOccChunk <= 32, "a chunk is staged one triangle per lane");
constexpr int kItemSamples = FDZB_OCC_ITEM;

// Row words: uint32_t (grids up to 32 x 32, the reference's U32) or
// unsigned long long (up to 64 x 64, the reference's template at T = U64).
template <class R> struct RowWord;
template <> struct RowWord<uint32_t> {
    static constexpr int kBits = 32;
    static constexpr int kWarps = 4;
    static constexpr int kMinBlocks = FDZB_OCC_MINBLOCKS;
    __device__ static int lowest(uint32_t v) { return __ffs(v) - 1; }
    __device__ static int popc(uint32_t v) { return __popc(v); }
    __device__ static uint32_t fullCols(const LightParams &L) { return L.full; }
    __device__ static uint32_t fullRows(const LightParams &L) { return (uint32_t)L.fullRows; }
};
template <> struct RowWord<unsigned long long> {
    static constexpr int kBits = 64;
    static constexpr int kWarps = 2;
    static constexpr int kMinBlocks = 5;
    __device__ static int lowest(unsigned long long v) { return __ffsll((long long)v) - 1; }
    __device__ static int popc(unsigned long long v) { return __popcll(v); }
    __device__ static unsigned long long fullCols(const LightParams &L) { return L.fullCols; }
    __device__ static unsigned long long fullRows(const LightParams &L) { return L.fullRows; }
};
typedef unsigned long long u64;

// K/Step5_2_shadowCalPerSample.inl:14-33, as the range of set columns.  With
// f1 = D >= 0, f2 = D + slope*(count-1) >= 0 and k = the round-up conversion
// of q (q = -D / slope rounded to nearest, as the reference divides; its
// truncating conversion of ceilf(q) is the same integer) the reference's mask
// is: all columns when f1 and f2, none when neither, else (1 << k) - 1 (PTX
// shl: amounts >= the word width give 0), complemented when !f1, limited to
// the grid.  In the partial cases 0 <= k <= count: D and D + slope*(count-1)
// have opposite signs, so |q| <= (count-1)(1 + 2^-24) and the quotient's sign
// is that of D / (D - (D + Bn)), i.e. q >= 0.  So the mask is the column range
// [lo, hi) with lo = f1 ? 0 : k and hi = f2 ? count : k -- [0, count) when
// both hold, [0, k) or [k, count) when one does, and [k, k) = nothing when
// neither (whatever k is then).  A row's mask, the AND of its edges' masks,
// is the intersection of their ranges: [max lo, min hi).  This replaces
// per-edge shifts, complements and selections by two min/max and one
// two-shift difference per row (measured: HD frame occlusion 6.48 -> 5.94
// ms, large frame 1457 -> 1290 ms).  npart counts the partial cases (COUNT).
template <int COUNT>
__device__ __forceinline__ void col_range(float D, float slopeNm1, float q, int count, int &lo, int &hi,
                                          uint32_t &npart)
{
    const bool f1 = D >= 0.0f;
    const bool f2 = __fadd_rn(slopeNm1, D) >= 0.0f;
    if (COUNT) npart += (f1 != f2);
    const int k = __float2int_ru(q);
    lo = f1 ? 0 : k;
    hi = f2 ? count : k;
}

// 1 << s with the PTX shl semantics (0 for s >= the word width; s < 0 read as
// unsigned, so 0 as well), and the bits [lo, hi) (none when hi <= lo).
template <class R> __device__ __forceinline__ R bit_at(int s);
template <> __device__ __forceinline__ uint32_t bit_at<uint32_t>(int s)
{
    return __funnelshift_lc(0u, 1u, (unsigned)s);   // high word of (1:0) << min(s, 32)
}
template <> __device__ __forceinline__ unsigned long long bit_at<unsigned long long>(int s)
{
    return (unsigned)s >= 64u ? 0ull : (1ull << s);
}
template <class R> __device__ __forceinline__ R range_bits(int lo, int hi)
{
    return bit_at<R>(max(hi, lo)) - bit_at<R>(lo);
}

// a / b rounded to nearest, from y = RN(1/b): two correction steps of
// Markstein's method (P. Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990, with the
// theorem as restated in Muller et al., Handbook of Floating-Point
// Arithmetic, sec. 4.7).  With a, b, y free of underflow and overflow:
// q0 = RN(a y) lies within two ulps of a/b, so each residual a - b q is exact
// (an FMA); the first step brings q within one ulp (in fact within half an
// ulp plus a term of order 2^-46), and the second, by Markstein's theorem (y
// within half an ulp of 1/b, q within one ulp of a/b), returns RN(a/b).  The
// pair test hoists y out of its row loop, one reciprocal per edge, so that a
// row's quotient costs five FP32 operations instead of a division; a device
// self-check (fdzb_check_division) compares it with the IEEE division.
__device__ __forceinline__ float div_by_rcp(float a, float b, float y)
{
    const float q0 = __fmul_rn(a, y);
    const float r0 = __fmaf_rn(-b, q0, a);
    const float q1 = __fmaf_rn(r0, y, q0);
    const float r1 = __fmaf_rn(-b, q1, a);
    return __fmaf_rn(r1, y, q1);
}

// RN(1/b) for normal b with |b| in [2^-100, 2^40): the hardware's approximate
// reciprocal (rcp.approx) and one Newton-Raphson step in FMA form,
// y1 = y0 + y0 (1 - b y0) (the iteration of Markstein's paper above and of
// Muller et al., sec. 4.7).  On that range the result equals the correctly
// rounded reciprocal (__frcp_rn) for every one of its 2^23 x 140 x 2 values,
// which the device self-check (fdzb_check_division) enumerates; the pair
// test uses it only there (elsewhere the row loop takes the IEEE division
// and ignores it).  Measured against __frcp_rn: HD frame 6.60 -> 6.35 ms.
__device__ __forceinline__ float rcp_nearest(float b)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(b));
    return __fmaf_rn(y, __fmaf_rn(-b, y, 1.0f), y);
}

// The same mask, over the light rows (the row filter, :176-191), with the
// full and empty cases returned before the division: the per-pair row
// filter's masks are mostly full or empty across the warp, so there the
// branch pays (measured: HD frame occlusion 6.88 -> 6.82 ms, 20k-triangle
// frame 7.52 -> 7.44 ms against a branch-free form).
template <class R, int COUNT>
__device__ __forceinline__ R row_filter_mask(float D, float slopeNm1, float slope, R full, uint32_t &npart)
{
    const bool f1 = D >= 0.0f;
    const bool f2 = __fadd_rn(slopeNm1, D) >= 0.0f;
    if (f1 && f2) return full;
    if (!f1 && !f2) return R(0);
    if (COUNT) ++npart;
    const float q = __fdiv_rn(-D, slope);
    const int k = __float2int_ru(q);
    R m = ((unsigned)k >= (unsigned)RowWord<R>::kBits) ? R(0) : (R(1) << k);
    m -= R(1);
    if (!f1) m = ~m;
    return m & full;
}

// K/Step5_2_shadowCal.inl:213-222
__device__ __forceinline__ bool point_in_tri(f3 A, f3 B, f3 C, f3 P)
{
    const f3 N1 = cross3(sub3(B, A), sub3(P, B));
    const f3 N2 = cross3(sub3(C, B), sub3(P, C));
    if (dot3(N1, N2) < 0.0f) return false;
    const f3 N3 = cross3(sub3(A, C), sub3(P, A));
    if (dot3(N2, N3) < 0.0f) return false;
    return true;
}

// Staged triangle, 7 x float4:
//  p0 = (aabb min x, min y, max x, max y)   p1 = (minz, v0)
//  p2 = (v1, v2.x)   p3 = (v2.y, v2.z, n.x, n.y)   p4 = (n.z, e01)
//  p5 = (e12, e20.x) p6 = (e20.y, e20.z, maxz, 0)
struct StagedTri {
    float4 p[7];
};

__device__ __forceinline__ void stage_triangle(StagedTri &dst, const float4 *__restrict__ rec, int tri)
{
    const float4 q0 = __ldg(rec + 4 * (size_t)tri);
    const float4 q1 = __ldg(rec + 4 * (size_t)tri + 1);
    const float4 q2 = __ldg(rec + 4 * (size_t)tri + 2);
    const float4 q3 = __ldg(rec + 4 * (size_t)tri + 3);
    const f3 v0 = mk3(q0.x, q0.y, q0.z), v1 = mk3(q1.x, q1.y, q1.z), v2 = mk3(q2.x, q2.y, q2.z);
    const f3 n = cross3(sub3(v1, v0), sub3(v2, v1));   // K/Step5_2_shadowCalPerSample.inl:130
    const f3 e01 = sub3(v0, v1), e12 = sub3(v1, v2), e20 = sub3(v2, v0);  // a - b of :7
    dst.p[0] = q3;
    dst.p[1] = make_float4(q0.w, v0.x, v0.y, v0.z);
    dst.p[2] = make_float4(v1.x, v1.y, v1.z, v2.x);
    dst.p[3] = make_float4(v2.y, v2.z, n.x, n.y);
    dst.p[4] = make_float4(n.z, e01.x, e01.y, e01.z);
    dst.p[5] = make_float4(e12.x, e12.y, e12.z, e20.x);
    dst.p[6] = make_float4(e20.y, e20.z, q1.w, 0.0f);
}

struct LaneSample {
    f3 Q, L0Q;
    float spx, spy, spz, spw, spZ;
};

// ---------------------------------------------------------------------------
// Open-box cull (lane per sample, edge-function masks).
//
// Seen from the light's upRight corner (the projection M of the light setup),
// a point X has u = M-projected x and depth w.  Light sample (r, c) lies at
// camera x = -r |x_delt|, depth 0, so a point P on the segment from light
// sample row r to the receiver Q satisfies u_P + k_r / w_P = u_Q + k_r / w_Q,
// k_r = RF.x r / (rows - 1) (RF.x = P00 (rows - 1) |x_delt| / 2, the
// reference's RectangleFactor).  For rows r in [r0, r1] it follows that some
// point of the triangle has u + k_r0 / w <= u_Q + k_r0 / w_Q and some point has
// u + k_r1 / w >= u_Q + k_r1 / w_Q; over a triangle in front of the light
// plane (every w > 0) u + k / w is linear-fractional, so its extremes are at
// the vertices.  The same holds for v and the columns.  With r0 = 0 and
// r1 = rows - 1 this is the reference's own pre-cull (the triangle's AABB
// against the sample's rectangle, K/Step5_2_shadowCalPerSample.inl:120-128).
//
// A sample's unset mask bits lie in a box: rows [r0, r1] (the rows not yet
// full) by columns [c0, c1] (the columns unset in some open row).  A pair
// whose triangle fails the test for that box, by a margin of 1e-3 of the
// sample's rectangle plus 1e-5, cannot set an unset bit: bits outside the box
// are set already, and inside it the pair's FP32 row masks could only set a
// bit within FP32 rounding (about 1e-7 of these coordinates) of the exact
// triangle boundary.  Skipping the pair leaves the mask -- the OR over the
// bin's triangles -- unchanged.  The box is refreshed at every staged chunk
// (a stale box is larger, so the test stays conservative), and triangles that
// reach the light plane (minz <= 0) are never skipped.  The union of the
// warp's boxes is also tested when a chunk is staged: a triangle no lane can
// use is skipped by the whole warp.
//
// The cull runs in its own instantiation of the kernel (BOX = 1): it pays where
// samples end in umbra (the HD frame: 43% fewer pair tests, 12% faster) and
// costs some 8% where most samples stay in penumbra (pair tests barely drop);
// the engine picks per launch (fdzb_api.cpp: open-box probe).
// ---------------------------------------------------------------------------
struct StagedPrj {
    float4 a, b;   // (u0, v0, 1/w0, u1), (v1, 1/w1, u2, v2)
    float c;       // 1/w2
};

// The vertices' projections, written by the triangle setup (k_tri_setup):
// prjRec holds (u0, v0, 1/w0, u1), (v1, 1/w1, u2, v2) and the record's third
// float4 carries 1/w2 in w.
__device__ __forceinline__ void stage_projection(StagedPrj &dst, const float4 *__restrict__ prjRec,
                                                 const float4 *__restrict__ rec, int tri)
{
    dst.a = __ldg(prjRec + 2 * (size_t)tri);
    dst.b = __ldg(prjRec + 2 * (size_t)tri + 1);
    dst.c = __ldg(rec + 4 * (size_t)tri + 2).w;
}

// A lane's open box as thresholds: (k_r0, k_r1, u_Q + k_r0/w_Q + mu, u_Q + k_r1/w_Q - mu)
// and the same for columns and v.
struct OpenBox {
    float4 u, v;
};

template <class R>
__device__ __forceinline__ int highest_bit(R v)
{
    return (int)(8 * sizeof(R)) - 1 - (sizeof(R) == 8 ? __clzll((long long)v) : __clz((int)v));
}

// Returns false when the box is the whole grid: the per-lane test would then
// repeat the reference's pre-cull (the box is still filled, for the union).
template <class R>
__device__ __forceinline__ bool open_box(OpenBox &box, const LaneSample &s, const LightParams &L, int NR, int NC,
                                        R FR, R FC, R fullRows, R (*rows)[32], int lane)
{
    const R orow = FR & ~fullRows;
    R ocol = 0;
    for (R m = orow; m; m &= m - R(1)) ocol |= ~rows[RowWord<R>::lowest(m)][lane];
    ocol &= FC;
    const bool whole = orow == FR && ocol == FC;
    if (!orow || !ocol) {
        // nothing open: every test fails (the walk ends at this chunk)
        box.u = make_float4(0.f, 0.f, -kF32Max, kF32Max);
        box.v = box.u;
        return true;
    }
    const float iwq = __frcp_rn(s.spZ);
    const int r0 = RowWord<R>::lowest(orow), r1 = highest_bit<R>(orow);
    const int c0 = RowWord<R>::lowest(ocol), c1 = highest_bit<R>(ocol);
    const float su = NR > 1 ? L.RF[0] / (float)(NR - 1) : 0.f, sv = NC > 1 ? L.RF[1] / (float)(NC - 1) : 0.f;
    const float ku0 = su * (float)r0, ku1 = su * (float)r1, kv0 = sv * (float)c0, kv1 = sv * (float)c1;
    const float mu = 1e-3f * L.RF[0] * iwq + 1e-5f, mv = 1e-3f * L.RF[1] * iwq + 1e-5f;
    box.u = make_float4(ku0, ku1, s.spx + ku0 * iwq + mu, s.spx + ku1 * iwq - mu);
    box.v = make_float4(kv0, kv1, s.spy + kv0 * iwq + mv, s.spy + kv1 * iwq - mv);
    return !whole;
}

// The union over the warp's active lanes of their boxes: a triangle that one
// lane's test passes passes the union's (smaller k and larger threshold on
// the min side, the reverse on the max side, since 1/w > 0), so a triangle the
// union test rejects is rejected by every lane's.
__device__ __forceinline__ OpenBox union_box(const OpenBox &b, bool active)
{
    float a0 = active ? b.u.x : kF32Max, a1 = active ? b.u.y : -kF32Max;
    float a2 = active ? b.u.z : -kF32Max, a3 = active ? b.u.w : kF32Max;
    float c0 = active ? b.v.x : kF32Max, c1 = active ? b.v.y : -kF32Max;
    float c2 = active ? b.v.z : -kF32Max, c3 = active ? b.v.w : kF32Max;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a0 = fminf(a0, __shfl_xor_sync(kFullWarp, a0, o));
        a1 = fmaxf(a1, __shfl_xor_sync(kFullWarp, a1, o));
        a2 = fmaxf(a2, __shfl_xor_sync(kFullWarp, a2, o));
        a3 = fminf(a3, __shfl_xor_sync(kFullWarp, a3, o));
        c0 = fminf(c0, __shfl_xor_sync(kFullWarp, c0, o));
        c1 = fmaxf(c1, __shfl_xor_sync(kFullWarp, c1, o));
        c2 = fmaxf(c2, __shfl_xor_sync(kFullWarp, c2, o));
        c3 = fminf(c3, __shfl_xor_sync(kFullWarp, c3, o));
    }
    OpenBox u;
    u.u = make_float4(a0, a1, a2, a3);
    u.v = make_float4(c0, c1, c2, c3);
    return u;
}

// The reference's pre-cull of a pair (K/Step5_2_shadowCalPerSample.inl:120-128).
__device__ __forceinline__ bool precull_pass(const StagedTri &T, const LaneSample &s)
{
    const float4 p0 = T.p[0];
    return p0.x <= s.spx && p0.y <= s.spy && s.spz <= p0.z && s.spw <= p0.w && T.p[1].x <= s.spZ;
}

// True if the triangle may set a bit inside the lane's open box.
__device__ __forceinline__ bool box_reach(const StagedPrj &P, const OpenBox &b)
{
    const float4 a = P.a, c = P.b;
    const float w2 = P.c;
    const float umin = fminf(fminf(__fmaf_rn(b.u.x, a.z, a.x), __fmaf_rn(b.u.x, c.y, a.w)), __fmaf_rn(b.u.x, w2, c.z));
    const float umax = fmaxf(fmaxf(__fmaf_rn(b.u.y, a.z, a.x), __fmaf_rn(b.u.y, c.y, a.w)), __fmaf_rn(b.u.y, w2, c.z));
    const float vmin = fminf(fminf(__fmaf_rn(b.v.x, a.z, a.y), __fmaf_rn(b.v.x, c.y, c.x)), __fmaf_rn(b.v.x, w2, c.w));
    const float vmax = fmaxf(fmaxf(__fmaf_rn(b.v.y, a.z, a.y), __fmaf_rn(b.v.y, c.y, c.x)), __fmaf_rn(b.v.y, w2, c.w));
    return umin <= b.u.z && umax >= b.u.w && vmin <= b.v.z && vmax >= b.v.w;
}

__device__ __forceinline__ void load_sample(LaneSample &s, const FrameDesc &fr, const FrameState &st,
                                            int local)
{
    const float4 P = __ldg(fr.pos + local);
    s.Q = mk3(P.x, P.y, P.z);
    const f3 r = light_project(fr.light.mat, s.Q);
    s.spx = r.x;
    s.spy = r.y;
    s.spz = __fsub_rn(__fadd_rn(r.x, __fdiv_rn(fr.light.RF[0], r.z)), st.subx);
    s.spw = __fsub_rn(__fadd_rn(r.y, __fdiv_rn(fr.light.RF[1], r.z)), st.suby);
    s.spZ = r.z;
    s.L0Q = sub3(ld3(fr.light.ur), s.Q);
}

// Light grid constants of a frame, in the form the pair tests use them.
template <class R> struct GridC {
    int NR, NC;             // rows (along x_delt), columns (along y_delt)
    float nrm1, ncm1;       // NR - 1, NC - 1
    R FR, FC;               // NR and NC low bits
};
template <class R> __device__ __forceinline__ GridC<R> grid_of(const FrameDesc &fr)
{
    GridC<R> g;
    g.NR = fr.light.N;
    g.NC = fr.light.NC;
    g.nrm1 = (float)(g.NR - 1);
    g.ncm1 = (float)(g.NC - 1);
    g.FR = RowWord<R>::fullRows(fr.light);
    g.FC = RowWord<R>::fullCols(fr.light);
    return g;
}

// One sample/triangle pair (K/Step5_2_shadowCalPerSample.inl:120-222).  Rows r
// step along x_delt (A), columns c along y_delt (B); the row filter bounds the
// column term with B*(NC-1) and the rows with A*(NR-1), which for the
// reference's square grids are its own expressions.  With the depth plane, a
// fourth plane -n.(L - v0), oriented like the edges, keeps light samples on
// the sample's side of the triangle unoccluded (the test of the reference's
// per-bin kernel, K/Step5_2_shadowCal.inl:667-674, 838) for triangles that
// reach the light plane (min depth <= 0: occluders behind the light) or the
// sample's depth (the per-bin kernel's own condition); a triangle strictly
// between them needs no such test.  Returns 1 if the pair passed the AABB
// pre-cull.  FLAT = 1 evaluates all three edges of every open row instead of
// stopping once the row mask holds nothing new (see the row loop).
// PRECULLED = 1: the caller has already found that the pair passes the
// pre-cull.
template <class R, int DEPTH, int FLAT, int COUNT, int PRECULLED>
__device__ __forceinline__ int pair_test(const StagedTri &T, const LaneSample &s, f3 xd, f3 yd, f3 ur,
                                         float esp, const GridC<R> &g, R (*rows)[32], int lane, R &fullRows,
                                         uint32_t &nrows, uint32_t &npart)
{
    const float4 p1 = T.p[1];
    if (!PRECULLED) {
        const float4 p0 = T.p[0];
        if (!(p0.x <= s.spx && p0.y <= s.spy && s.spz <= p0.z && s.spw <= p0.w && p1.x <= s.spZ)) return 0;
    }
    const float4 p2 = T.p[2], p3 = T.p[3], p4 = T.p[4], p5 = T.p[5], p6 = T.p[6];
    const f3 v0 = mk3(p1.y, p1.z, p1.w), v1 = mk3(p2.x, p2.y, p2.z), v2 = mk3(p2.w, p3.x, p3.y);
    const f3 n = mk3(p3.z, p3.w, p4.x);
    const f3 e01 = mk3(p4.y, p4.z, p4.w), e12 = mk3(p5.x, p5.y, p5.z), e20 = mk3(p5.w, p6.x, p6.y);
    const f3 Q = s.Q;
    const float dir = dot3(sub3(Q, v0), n);
    if (fabsf(dir) < esp && point_in_tri(v0, v1, v2, Q)) return 1;
    // orientation: the reference negates t0, t1 and L0 - Q when dir < 0
    const bool neg = dir < 0.0f;
    const f3 t0 = neg ? mk3(-xd.x, -xd.y, -xd.z) : xd;
    const f3 t1 = neg ? mk3(-yd.x, -yd.y, -yd.z) : yd;
    const f3 lq = neg ? mk3(-s.L0Q.x, -s.L0Q.y, -s.L0Q.z) : s.L0Q;
    // getPlaneDiscriminant for (v0,v1), (v1,v2), (v2,v0): n_k = cross(b - Q, a - b)
    const f3 n0 = cross3(sub3(v1, Q), e01);
    const f3 n1 = cross3(sub3(v2, Q), e12);
    const f3 n2 = cross3(sub3(v0, Q), e20);
    const float A0 = dot3(n0, t0), B0 = dot3(n0, t1), C0 = dot3(n0, lq);
    const float A1 = dot3(n1, t0), B1 = dot3(n1, t1), C1 = dot3(n1, lq);
    const float A2 = dot3(n2, t0), B2 = dot3(n2, t1), C2 = dot3(n2, lq);
    const float An0 = __fmul_rn(A0, g.nrm1), An1 = __fmul_rn(A1, g.nrm1), An2 = __fmul_rn(A2, g.nrm1);
    const float Bn0 = __fmul_rn(B0, g.ncm1), Bn1 = __fmul_rn(B1, g.ncm1), Bn2 = __fmul_rn(B2, g.ncm1);
    // row filter (:176-191)
    const R N0 = row_filter_mask<R, COUNT>(__fadd_rn(B0 > 0.0f ? Bn0 : 0.0f, C0), An0, A0, g.FR, npart);
    const R N1 = row_filter_mask<R, COUNT>(__fadd_rn(B1 > 0.0f ? Bn1 : 0.0f, C1), An1, A1, g.FR, npart);
    const R N2 = row_filter_mask<R, COUNT>(__fadd_rn(B2 > 0.0f ? Bn2 : 0.0f, C2), An2, A2, g.FR, npart);
    R vr = N0 & N1 & N2 & ~fullRows;
    const bool dp = DEPTH && (p1.x <= 0.0f || p6.z >= s.spZ);
    float A3 = 0.0f, B3 = 0.0f, C3 = 0.0f, Bn3 = 0.0f;
    if (dp && vr) {
        const f3 m = mk3(-n.x, -n.y, -n.z);
        const f3 lv0 = sub3(ur, v0);
        const f3 lv = neg ? mk3(-lv0.x, -lv0.y, -lv0.z) : lv0;
        A3 = dot3(m, t0);
        B3 = dot3(m, t1);
        C3 = dot3(m, lv);
        Bn3 = __fmul_rn(B3, g.ncm1);
        vr &= row_filter_mask<R, COUNT>(__fadd_rn(B3 > 0.0f ? Bn3 : 0.0f, C3), __fmul_rn(A3, g.nrm1), A3, g.FR, npart);
    }
    // The rows' quotients -D / B_k by div_by_rcp with y_k = RN(1/B_k).  Its
    // preconditions hold when every A_k and C_k lies in [2^-38, 2^40] and every
    // B_k in [2^-100, 2^39] (magnitudes): then D = RN(RN(A_k r) + C_k) is a
    // multiple of 2^-61 (each term is a multiple of its operand's ulp), so a
    // nonzero D has |D| >= 2^-61 and |D| <= 2^47; a partial row (D and
    // D + B_k (count-1) of opposite signs) has |D / B_k| < 64, and with
    // |B_k| <= 2^39 a nonzero quotient is at least 2^-100 -- no quantity of
    // the method underflows or overflows.  A zero D gives a zero quotient of
    // the division's sign either way.  Where the full and empty cases
    // discard the quotient, its value does not matter.  A pair outside these
    // ranges (a zero coefficient included) takes the IEEE division.
    // Measured: HD frame occlusion 6.82 -> 6.39 ms, 20k-triangle frame 7.46 ->
    // 6.85 ms, identical masks.
    const float lo = fminf(fminf(fminf(fabsf(A0), fabsf(A1)), fminf(fabsf(A2), fabsf(C0))),
                           fminf(fabsf(C1), fabsf(C2)));
    const float hi = fmaxf(fmaxf(fmaxf(fabsf(A0), fabsf(A1)), fmaxf(fabsf(A2), fabsf(C0))),
                           fmaxf(fabsf(C1), fabsf(C2)));
    const float bl = fminf(fminf(fabsf(B0), fabsf(B1)), fabsf(B2));
    const float bh = fmaxf(fmaxf(fabsf(B0), fabsf(B1)), fabsf(B2));
    const bool viaRcp = lo >= 0x1p-38f && hi <= 0x1p40f && bl >= 0x1p-100f && bh <= 0x1p39f;
    const float y0 = rcp_nearest(B0), y1 = rcp_nearest(B1), y2 = rcp_nearest(B2);
    // rows (:204-222).  The row's mask is the AND of the edges' masks, so it only
    // loses bits as edges are added: once it holds no bit the row lacks, the
    // remaining edges cannot change the row.  Without FLAT they are then not
    // evaluated; with it every edge is (no divergent branch per edge).  The
    // row is written back either way (OR-ing nothing new leaves it as it is).
    // Measured, the flat form pays in the open-box instantiation (HD frame
    // occlusion 7.09 -> 6.91 ms) and the early stop in the other (20k-triangle
    // frame 7.54 vs 7.62 ms); the unconditional write-back pays in the second
    // only when combined with the early stop.
    auto row_loop = [&](auto rcp) {
        constexpr bool kRcp = decltype(rcp)::value;
        auto quot = [&](float D, float B, float y) { return kRcp ? div_by_rcp(-D, B, y) : __fdiv_rn(-D, B); };
        while (vr) {
            const int r = RowWord<R>::lowest(vr);
            vr &= vr - R(1);
            if (COUNT) ++nrows;
            const float fr = (float)r;
            const R have = rows[r][lane];
            const float D0 = __fadd_rn(__fmul_rn(A0, fr), C0);
            int lo, hi;
            col_range<COUNT>(D0, Bn0, quot(D0, B0, y0), g.NC, lo, hi, npart);
            R m;
            if (FLAT) {
                const float D1 = __fadd_rn(__fmul_rn(A1, fr), C1);
                const float D2 = __fadd_rn(__fmul_rn(A2, fr), C2);
                int lo1, hi1, lo2, hi2;
                col_range<COUNT>(D1, Bn1, quot(D1, B1, y1), g.NC, lo1, hi1, npart);
                col_range<COUNT>(D2, Bn2, quot(D2, B2, y2), g.NC, lo2, hi2, npart);
                lo = max(lo, max(lo1, lo2));
                hi = min(hi, min(hi1, hi2));
                m = range_bits<R>(lo, hi);
            } else {
                m = range_bits<R>(lo, hi);
                if (m & ~have) {
                    const float D1 = __fadd_rn(__fmul_rn(A1, fr), C1);
                    int lo1, hi1;
                    col_range<COUNT>(D1, Bn1, quot(D1, B1, y1), g.NC, lo1, hi1, npart);
                    lo = max(lo, lo1);
                    hi = min(hi, hi1);
                    m = range_bits<R>(lo, hi);
                }
                if (m & ~have) {
                    const float D2 = __fadd_rn(__fmul_rn(A2, fr), C2);
                    int lo2, hi2;
                    col_range<COUNT>(D2, Bn2, quot(D2, B2, y2), g.NC, lo2, hi2, npart);
                    lo = max(lo, lo2);
                    hi = min(hi, hi2);
                    m = range_bits<R>(lo, hi);
                }
            }
            if (dp && (m & ~have)) {
                const float D3 = __fadd_rn(__fmul_rn(A3, fr), C3);
                int lo3, hi3;
                col_range<COUNT>(D3, Bn3, __fdiv_rn(-D3, B3), g.NC, lo3, hi3, npart);
                m = range_bits<R>(max(lo, lo3), min(hi, hi3));
            }
            const R nv = have | m;
            rows[r][lane] = nv;
            if (nv == g.FC) fullRows |= R(1) << r;
        }
    };
    if (viaRcp) row_loop(std::true_type{});
    else row_loop(std::false_type{});
    return 1;
}

// Ray-cast pair test: the reference's REF_CAL cross-check (refCal_kernel and
// intersect_triangle_branchless, K/Step5_2_calRef.inl:1-126).  For every light
// sample not yet occluded, a ray from the sample's position to the light
// sample's position; occluded when it meets the triangle with 1e-3 < t < dist.
// The reference numbers light sample (i along the light's height, j along its
// width) as i*W + j and places it at upRight + x_delt*j + y_delt*i
// (FS/api.cpp:351-357); here it is stored in this library's mask layout, row
// r = j (width), column c = i (height), so that the ray-cast and edge-function
// masks compare bit for bit.  Same pre-cull as the reference's checker: the
// sample's rectangle inside the triangle's AABB and minz - 1e-3 (in double, as
// the reference's double literal makes it) not above the sample's depth.
template <class R, int COUNT>
__device__ __forceinline__ int raycast_pair(const StagedTri &T, const LaneSample &s, f3 ur, f3 xd, f3 yd,
                                            const GridC<R> &g, R (*rows)[32], int lane, R &fullRows,
                                            uint32_t &nrows)
{
    const float4 p0a = T.p[0];
    const float4 p1a = T.p[1];
    if (!(s.spz <= p0a.z && s.spw <= p0a.w && s.spx >= p0a.x && s.spy >= p0a.y)) return 0;
    if ((double)p1a.x - 1e-3 > (double)s.spZ) return 0;
    const float4 p2a = T.p[2], p3a = T.p[3];
    const f3 v0 = mk3(p1a.y, p1a.z, p1a.w), v1 = mk3(p2a.x, p2a.y, p2a.z), v2 = mk3(p2a.w, p3a.x, p3a.y);
    const f3 e0 = sub3(v1, v0);
    const f3 e1 = sub3(v0, v2);
    const f3 n = cross3(e1, e0);
    const f3 q0 = sub3(v0, s.Q);
    const float tmin = 1e-3f;
    for (int r = 0; r < g.NR; ++r) {
        const R have = rows[r][lane];
        if (have == g.FC) continue;
        if (COUNT) ++nrows;
        const f3 lr = add3(ur, mul3(xd, (float)r));   // upRight + x_delt * j
        R add = 0;
        for (int c = 0; c < g.NC; ++c) {
            if (have & (R(1) << c)) continue;
            const f3 lp = add3(lr, mul3(yd, (float)c));   // ... + y_delt * i
            const f3 L = sub3(lp, s.Q);
            const float dist = __fsqrt_rn(dot3(L, L));
            const f3 dir = mk3(__fdiv_rn(L.x, dist), __fdiv_rn(L.y, dist), __fdiv_rn(L.z, dist));
            const float inv = __fdiv_rn(1.0f, dot3(n, dir));
            const f3 e2 = mul3(q0, inv);
            const f3 iv = cross3(dir, e2);
            const float beta = dot3(iv, e1);
            const float gamma = dot3(iv, e0);
            const float t = dot3(n, e2);
            if ((t < dist) & (t > tmin) & (beta >= 0.0f) & (gamma >= 0.0f) & (__fadd_rn(beta, gamma) <= 1.0f))
                add |= R(1) << c;
        }
        if (add) {
            const R nv = have | add;
            rows[r][lane] = nv;
            if (nv == g.FC) fullRows |= R(1) << r;
        }
    }
    return 1;
}

// Bits [pos, pos + n) of a packed mask (n <= 64), LSB first.
__device__ __forceinline__ u64 mask_bits(const uint32_t *w, int pos, int n)
{
    u64 v = 0;
    int got = 0;
    while (got < n) {
        const int wi = (pos + got) >> 5, o = (pos + got) & 31;
        const int take = min(32 - o, n - got);
        const uint32_t part = (w[wi] >> o) & (take == 32 ? 0xffffffffu : ((1u << take) - 1u));
        v |= (u64)part << got;
        got += take;
    }
    return v;
}

// Shadow = set bits / (rows * cols) (:226-231) and the packed mask, bit r * NC + c.
template <class R>
__device__ __forceinline__ void write_result(const FrameDesc &fr, int local, const GridC<R> &g, R (*rows)[32],
                                             int lane)
{
    int cnt = 0;
    for (int r = 0; r < g.NR; ++r) cnt += RowWord<R>::popc(rows[r][lane]);
    fr.shadow[local] = __fdiv_rn((float)cnt, (float)(g.NR * g.NC));   // :226-231
    if (fr.masks) {
        uint32_t *mo = fr.masks + (size_t)local * fr.maskWords;
        u64 acc = 0;
        int bit = 0, wi = 0;
        for (int r = 0; r < g.NR; ++r) {
            u64 v = (u64)rows[r][lane];
            int rem = g.NC;
            while (rem > 0) {
                const int take = min(rem, 32);
                const u64 part = v & (take == 32 ? 0xffffffffull : ((1ull << take) - 1ull));
                acc |= part << bit;
                bit += take;
                if (bit >= 32) {
                    mo[wi++] = (uint32_t)acc;
                    acc >>= 32;
                    bit -= 32;
                }
                v >>= take;
                rem -= take;
            }
        }
        if (bit > 0) mo[wi] = (uint32_t)acc;
    }
}

// Rows of a sample from its packed mask (bit r*NC + c is row r, column c), for
// a launch that accumulates into masks of an earlier triangle pass.  Returns
// the set of full rows.
template <class R>
__device__ __forceinline__ R load_rows(const FrameDesc &fr, int local, const GridC<R> &g, R (*rows)[32], int lane)
{
    const uint32_t *mi = fr.masks + (size_t)local * fr.maskWords;
    R fullRows = 0;
    for (int r = 0; r < g.NR; ++r) {
        const R v = (R)mask_bits(mi, r * g.NC, g.NC) & g.FC;
        rows[r][lane] = v;
        if (v == g.FC) fullRows |= R(1) << r;
    }
    return fullRows;
}

// First contact of a sample with the pipeline's occlusion stage: rows cleared,
// or loaded from the masks of an earlier triangle pass.
template <class R>
__device__ __forceinline__ R init_rows(const FrameDesc &fr, int local, const GridC<R> &g, R (*rows)[32], int lane)
{
    if (fr.accumulate) return load_rows<R>(fr, local, g, rows, lane);
    for (int r = 0; r < g.NR; ++r) rows[r][lane] = 0;
    return 0;
}

__device__ __forceinline__ void write_zero(const FrameDesc &fr, int local)
{
    fr.shadow[local] = 0.0f;
    if (fr.masks) {
        uint32_t *mo = fr.masks + (size_t)local * fr.maskWords;
        for (int w = 0; w < fr.maskWords; ++w) mo[w] = 0u;
    }
}

// Samples per work item of a frame (FrameDesc::occItem; 32 if out of range).
__device__ __forceinline__ int item_samples(const FrameDesc &fr)
{
    const int v = fr.occItem;
    return (v == 64 || v == 128) ? v : kItemSamples;
}

// Triangles staged per chunk of a frame (FrameDesc::occChunk, within [1, kOccChunk]).
__device__ __forceinline__ int chunk_of(const FrameDesc &fr)
{
    const int v = fr.occChunk;
    return (v >= 1 && v <= kOccChunk) ? v : kOccChunk;
}

// k_items: one thread per bin; a bin with n samples yields ceil(n / item) items
// (bin, first sample offset, frame, triangle count), item = the frame's samples
// per work item.
__global__ void k_items(const FrameDesc *__restrict__ frames, int32_t *__restrict__ bss,
                        int32_t *__restrict__ bse, int32_t *__restrict__ bts,
                        int32_t *__restrict__ bte, const int *__restrict__ binBases, int nframes,
                        int totalBins, int4 *__restrict__ items, int capacity, Counters *ctr)
{
    const int lane = threadIdx.x & 31;
    // segments no element reached hold (kSegAbsent, 0): (0, 0), as the
    // reference's pre-zeroed arrays (the samples' array has the extra slot of
    // the unbinned samples)
    if (blockIdx.x == 0 && threadIdx.x == 0 && bss[totalBins] == kSegAbsent) bss[totalBins] = bse[totalBins] = 0;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < totalBins;
         base += gridDim.x * blockDim.x) {
        const int b = base + lane;
        int n = 0, f = 0, isz = kItemSamples;
        if (b < totalBins) {
            if (bss[b] == kSegAbsent) bss[b] = bse[b] = 0;
            if (bts[b] == kSegAbsent) bts[b] = bte[b] = 0;
            const int cnt = bse[b] - bss[b];
            if (cnt > 0) {
                f = frame_of(binBases, nframes, b);
                isz = item_samples(frames[f]);
                n = (cnt + isz - 1) / isz;
            }
        }
        int x = n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFullWarp, x, o);
            if (lane >= o) x += y;
        }
        const int tot = __shfl_sync(kFullWarp, x, 31);
        int wbase = 0;
        if (lane == 0 && tot) wbase = atomicAdd(&ctr->itemCount, tot);
        wbase = __shfl_sync(kFullWarp, wbase, 0);
        if (n) {
            const int nt = bte[b] - bts[b];
            for (int k = 0; k < n; ++k) {
                const int slot = wbase + x - n + k;
                if (slot < capacity) items[slot] = make_int4(b, isz * k, f, nt);
            }
        }
    }
}

// RAYCAST = 1: the ray-cast cross-check instead of the edge-function masks.
// R: the row word (uint32_t for grids up to 32 x 32, u64 up to 64 x 64; the
// 64-bit form runs 2 warps per block to keep its rows in shared memory).
// DEPTH = 1: the edge-function masks also test the triangle's own plane.
// BOX = 1: the open-box cull (edge-function masks only).
// COUNT = 1: the work counters (pair tests, light rows, partial row masks) are
// accumulated; the engine runs this form when profiling is on.  Counting costs
// an add per row and per edge, 4-6 % of the kernel (measured); the open-box
// cull's own counters (skipped and examined pairs) are kept in both forms.
// ROWS: light rows a lane's mask holds in shared memory (RowWord<R>::kBits, or
// 16 for launches whose grids have at most 16 rows: the open-box form then
// takes 28.7 KB of shared memory a block instead of 36.9 KB and 7 blocks fit
// an SM instead of 6 -- HD frame 6.21 -> 6.08 ms).
template <int RAYCAST, class R, int DEPTH, int BOX, int COUNT, int ROWS = RowWord<R>::kBits>
__global__ void __launch_bounds__(RowWord<R>::kWarps * 32, RowWord<R>::kMinBlocks)
    k_occlusion(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ states,
                const int4 *__restrict__ items, int itemCapacity, Counters *ctr,
                const uint32_t *__restrict__ sortedVals, const int32_t *__restrict__ bss,
                const int32_t *__restrict__ bse, const int32_t *__restrict__ bts,
                const int32_t *__restrict__ bte, const uint32_t *__restrict__ pairTri, uint32_t triMask,
                const float4 *__restrict__ rec, const float4 *__restrict__ prjRec, int totalTris, int totalBins,
                int nframes)
{
    __shared__ StagedTri s_tri[RowWord<R>::kWarps][kOccChunk];
    static_assert(ROWS >= 1 && ROWS <= RowWord<R>::kBits, "rows of a lane's mask");
    __shared__ R s_rows[RowWord<R>::kWarps][ROWS][32];
    constexpr bool kRefine = BOX && !RAYCAST;
    __shared__ StagedPrj s_prj[kRefine ? RowWord<R>::kWarps : 1][kRefine ? kOccChunk : 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    R(*rows)[32] = s_rows[warp];
    StagedTri *tris = s_tri[warp];
    StagedPrj *prj = s_prj[kRefine ? warp : 0];
    unsigned long long boxSkips = 0, examined = 0;
    unsigned long long tested = 0;
    uint32_t nrows = 0, npart = 0;
    int nitems = *(volatile const int *)&ctr->itemCount;
    if (nitems > itemCapacity) nitems = itemCapacity;

    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(&ctr->itemCursor, 1);
        it = __shfl_sync(kFullWarp, it, 0);
        if (it >= nitems) break;
        const int4 item = items[it];
        const int bin = item.x, fi = item.z;
        if ((unsigned)bin >= (unsigned)totalBins || (unsigned)fi >= (unsigned)nframes) {
            if (lane == 0) atomicOr(&ctr->errorFlags, (int)ERR_INTERNAL);
            continue;
        }
        const FrameDesc &fr = frames[fi];
        const FrameState &st = states[fi];
        const int S = fr.W * fr.H;
        const int sLo = bss[bin] + item.y;
        const int sHi = min(sLo + item_samples(fr), bse[bin]);
        const int tS = bts[bin];
        const int nT = bte[bin] - tS;
        const int chunk = chunk_of(fr);

        if (nT <= 0) {
            // no triangle in this bin: shadow 0 -- or, in a later triangle pass,
            // the result of the earlier passes, left as it is
            if (!fr.accumulate) {
                for (int k = sLo + lane; k < sHi; k += 32) {
                    const int local = (int)sortedVals[k] - fr.sampleBase;
                    if ((unsigned)local < (unsigned)S) write_zero(fr, local);
                    else atomicOr(&ctr->errorFlags, (int)ERR_INTERNAL);
                }
            }
            continue;
        }

        const GridC<R> g = grid_of<R>(fr);
        if (g.NR > ROWS) {   // the host picks ROWS from the launch's largest grid
            if (lane == 0) atomicOr(&ctr->errorFlags, (int)ERR_INTERNAL);
            continue;
        }
        const f3 xd = ld3(fr.light.xd), yd = ld3(fr.light.yd), ur = ld3(fr.light.ur);
        const float esp = fr.esp;

        LaneSample smp;
        OpenBox box;
        bool boxOn = false;
        int local = 0;
        int remaining = 0;
        R fullRows = 0;
        bool active = false;
        int next = sLo;
        // first fill
        {
            const int k = next + lane;
            if (k < sHi) {
                local = (int)sortedVals[k] - fr.sampleBase;
                if ((unsigned)local >= (unsigned)S) {
                    atomicOr(&ctr->errorFlags, (int)ERR_INTERNAL);
                } else {
                    active = true;
                    remaining = nT;
                    load_sample(smp, fr, st, local);
                    fullRows = init_rows<R>(fr, local, g, rows, lane);
                    if (fullRows == g.FR) remaining = 0;
                }
            }
            next += 32;
        }
        int cur = 0;  // offset of the next staged chunk within the bin's list
        while (__any_sync(kFullWarp, active)) {
            const int m = min(chunk, nT);
            __syncwarp();
            if (lane < m) {
                int off = cur + lane;
                if (off >= nT) off -= nT;
                int tri = (int)(pairTri[tS + off] & triMask);
                if ((unsigned)tri >= (unsigned)totalTris) {
                    atomicOr(&ctr->errorFlags, (int)ERR_INTERNAL);
                    tri = 0;
                }
                stage_triangle(tris[lane], rec, tri);
                if (kRefine) stage_projection(prj[lane], prjRec, rec, tri);
            }
            if (kRefine && remaining > 0)
                boxOn = open_box<R>(box, smp, fr.light, g.NR, g.NC, g.FR, g.FC, fullRows, rows, lane);
            __syncwarp();
            // staged triangle t against the lane's sample
            auto test_one = [&](int t) {
                if (RAYCAST) {
                    const int ts = raycast_pair<R, COUNT>(tris[t], smp, ur, xd, yd, g, rows, lane, fullRows, nrows);
                    if (COUNT) tested += ts;
                } else if (kRefine && !precull_pass(tris[t], smp)) {
                    // fails the reference's pre-cull: not a pair test (tested once, first,
                    // so that the box test runs only on pairs that pass it: HD frame
                    // 6.23 -> 6.18 ms)
                } else if (kRefine && boxOn && tris[t].p[1].x > 0.0f && !box_reach(prj[t], box)) {
                    ++boxSkips;
                } else {
                    const int ts = pair_test<R, DEPTH, kRefine, COUNT, kRefine>(tris[t], smp, xd, yd, ur, esp, g,
                                                                                rows, lane, fullRows, nrows, npart);
                    if (COUNT) tested += ts;
                }
                if (fullRows == g.FR) remaining = 0;
            };
            if (kRefine) {
                // triangles of the chunk that no active lane's box can use are
                // skipped by the whole warp (each lane would skip them anyway);
                // a lane's cycle covers the chunk's first rem0 triangles
                const int rem0 = remaining;
                const OpenBox ub = union_box(box, remaining > 0);
                const bool k = lane < m && (tris[lane].p[1].x <= 0.0f || box_reach(prj[lane], ub));
                const unsigned keep = __ballot_sync(kFullWarp, k);
                if (remaining > 0) {
                    // the lane's share of the chunk, and how much of it the union skips
                    const int own = rem0 < m ? rem0 : m;
                    const unsigned first = own >= 32 ? kFullWarp : ((1u << own) - 1u);
                    examined += (unsigned)own;
                    boxSkips += (unsigned)__popc(first & ~keep);
                }
                for (unsigned km = keep; km; km &= km - 1u) {
                    const int t = __ffs(km) - 1;
#if FDZB_OCC_VOTE
                    if (!__any_sync(kFullWarp, remaining > 0 && t < rem0)) break;
#endif
                    if (remaining > 0 && t < rem0) test_one(t);
                }
                if (remaining > 0) remaining = rem0 > m ? rem0 - m : 0;
            } else {
                for (int t = 0; t < m; ++t) {
#if FDZB_OCC_VOTE
                    if (!__any_sync(kFullWarp, remaining > 0)) break;
#endif
                    if (remaining > 0) {
                        --remaining;
                        test_one(t);
                    }
                }
            }
            cur += m;
            if (cur >= nT) cur -= nT;
            // retire finished lanes, then refill them with the item's next samples
            if (active && remaining == 0) {
                write_result<R>(fr, local, g, rows, lane);
                active = false;
            }
            const unsigned freeLanes = __ballot_sync(kFullWarp, !active);
#if FDZB_OCC_REFILL
            const bool refill = next < sHi && freeLanes;
#else
            // refill only once the whole batch is done, restarting at the head of
            // the (depth-ordered) list
            const bool refill = next < sHi && freeLanes == kFullWarp;
            if (refill) cur = 0;
#endif
            if (refill) {
                const int k = next + __popc(freeLanes & lanemask_lt());
                if (!active && k < sHi) {
                    local = (int)sortedVals[k] - fr.sampleBase;
                    if ((unsigned)local >= (unsigned)S) {
                        atomicOr(&ctr->errorFlags, (int)ERR_INTERNAL);
                    } else {
                        active = true;
                        remaining = nT;
                        load_sample(smp, fr, st, local);
                        fullRows = init_rows<R>(fr, local, g, rows, lane);
                        if (fullRows == g.FR) remaining = 0;
                    }
                }
                next += __popc(freeLanes);
            }
        }
    }
    unsigned long long t = tested, tr = nrows, tp = npart, tb = boxSkips, te = examined;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        t += __shfl_xor_sync(kFullWarp, t, o);
        tr += __shfl_xor_sync(kFullWarp, tr, o);
        tp += __shfl_xor_sync(kFullWarp, tp, o);
        tb += __shfl_xor_sync(kFullWarp, tb, o);
        te += __shfl_xor_sync(kFullWarp, te, o);
    }
    if (COUNT && lane == 0 && t) {
        atomicAdd(&ctr->pairTests, t);
        atomicAdd(&ctr->rowsEvaluated, tr);
        atomicAdd(&ctr->partialMasks, tp);
    }
    if (lane == 0 && tb) atomicAdd(&ctr->boxSkips, tb);
    if (lane == 0 && te) atomicAdd(&ctr->pairsExamined, te);
}


// ---------------------------------------------------------------------------
// k_occlusion_pairs: the same pair tests, scheduled so that every lane of a
// warp works on a pair that passed the AABB pre-cull.
//
// A warp owns a work item (up to 32 samples of one bin, one per lane, as in
// k_occlusion) and walks the bin's triangle list in chunks of kOccChunk staged
// triangles.  Per chunk:
//  1. cull: every lane tests its sample against each staged triangle's AABB and
//     minimum depth (the reference's pre-cull, K/Step5_2_shadowCalPerSample.inl
//     :120-128); a ballot per triangle gives the samples that pass it, and lane
//     t keeps the mask of triangle t;
//  2. compute: the passing pairs, numbered triangle-major through a warp scan
//     of the masks' popcounts, are dealt 32 at a time, one per lane; a lane
//     finds its pair's triangle by binary search over the scan, its sample as
//     the k-th set bit of that triangle's mask, fetches the sample's point from
//     the owning lane by shuffle and computes the pair's edge coefficients and
//     row filter;
//  3. rows: the (pair, light row) units of those 32 pairs are dealt 32 at a
//     time the same way; each lane evaluates the three row masks of its unit
//     (coefficients fetched from the pair's lane by shuffle) and ORs them into
//     the sample's row in shared memory by an atomic.
// A sample whose light rows are all full stops taking part (the reference's
// early-out); the pairs it still had in the chunk being dealt are skipped at
// their start.  The final mask is the OR over the bin's triangles either way.
// ---------------------------------------------------------------------------

#ifndef FDZB_OCC2_MINBLOCKS
#define FDZB_OCC2_MINBLOCKS 6
#endif

// Bit position of the k-th (0-based) set bit of m; k < popc(m).
__device__ __forceinline__ int nth_set_bit(uint32_t m, int k)
{
    int pos = 0;
    int c = __popc(m & 0xffffu);
    if (k >= c) { k -= c; pos += 16; m >>= 16; }
    c = __popc(m & 0xffu);
    if (k >= c) { k -= c; pos += 8; m >>= 8; }
    c = __popc(m & 0xfu);
    if (k >= c) { k -= c; pos += 4; m >>= 4; }
    c = __popc(m & 0x3u);
    if (k >= c) { k -= c; pos += 2; m >>= 2; }
    c = (int)(m & 1u);
    if (k >= c) pos += 1;
    return pos;
}

// The reference's row mask without branches: the threshold is computed
// whatever the case and selected away when the row is full or empty (the same
// mask as col_range's column range).
__device__ __forceinline__ uint32_t row_mask_sel(float D, float slopeNm1, float slope, uint32_t full,
                                                 uint32_t &npart)
{
    const bool f1 = D >= 0.0f;
    const bool f2 = __fadd_rn(slopeNm1, D) >= 0.0f;
    const float q = __fdiv_rn(-D, slope);
    const int k = __float2int_ru(q);
    uint32_t m = ((unsigned)k >= 32u) ? 0u : (1u << k);
    m -= 1u;
    m = f1 ? m : ~m;
    npart += (f1 != f2) ? 1u : 0u;
    m = (f1 == f2) ? (f1 ? full : 0u) : m;
    return m & full;
}

// Edge coefficients of one pair (K/Step5_2_shadowCalPerSample.inl:129-191): the
// light rows still open after the row filter, or 0 (self-skip, or nothing).
struct PairEdges {
    float A[3], B[3], C[3], Bn[3];
};

__device__ __forceinline__ uint32_t pair_setup(const StagedTri &T, f3 Q, f3 L0Q, f3 xd, f3 yd, float esp,
                                               float nm1, uint32_t FULL, uint32_t fullRows, PairEdges &e,
                                               uint32_t &npart)
{
    const float4 p1 = T.p[1], p2 = T.p[2], p3 = T.p[3], p4 = T.p[4], p5 = T.p[5], p6 = T.p[6];
    const f3 v0 = mk3(p1.y, p1.z, p1.w), v1 = mk3(p2.x, p2.y, p2.z), v2 = mk3(p2.w, p3.x, p3.y);
    const f3 n = mk3(p3.z, p3.w, p4.x);
    const f3 e01 = mk3(p4.y, p4.z, p4.w), e12 = mk3(p5.x, p5.y, p5.z), e20 = mk3(p5.w, p6.x, p6.y);
    const float dir = dot3(sub3(Q, v0), n);
    if (fabsf(dir) < esp && point_in_tri(v0, v1, v2, Q)) return 0u;
    const bool neg = dir < 0.0f;
    const f3 t0 = neg ? mk3(-xd.x, -xd.y, -xd.z) : xd;
    const f3 t1 = neg ? mk3(-yd.x, -yd.y, -yd.z) : yd;
    const f3 lq = neg ? mk3(-L0Q.x, -L0Q.y, -L0Q.z) : L0Q;
    const f3 n0 = cross3(sub3(v1, Q), e01);
    const f3 n1 = cross3(sub3(v2, Q), e12);
    const f3 n2 = cross3(sub3(v0, Q), e20);
    e.A[0] = dot3(n0, t0); e.B[0] = dot3(n0, t1); e.C[0] = dot3(n0, lq);
    e.A[1] = dot3(n1, t0); e.B[1] = dot3(n1, t1); e.C[1] = dot3(n1, lq);
    e.A[2] = dot3(n2, t0); e.B[2] = dot3(n2, t1); e.C[2] = dot3(n2, lq);
    uint32_t vr = FULL & ~fullRows;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float An = __fmul_rn(e.A[k], nm1);
        e.Bn[k] = __fmul_rn(e.B[k], nm1);
        vr &= row_mask_sel(__fadd_rn(e.B[k] > 0.0f ? e.Bn[k] : 0.0f, e.C[k]), An, e.A[k], FULL, npart);
    }
    return vr;
}

__global__ void __launch_bounds__(kOccThreads, FDZB_OCC2_MINBLOCKS)
    k_occlusion_pairs(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ states,
                      const int4 *__restrict__ items, int itemCapacity, Counters *ctr,
                      const uint32_t *__restrict__ sortedVals, const int32_t *__restrict__ bss,
                      const int32_t *__restrict__ bse, const int32_t *__restrict__ bts,
                      const int32_t *__restrict__ bte, const uint32_t *__restrict__ pairTri, uint32_t triMask,
                      const float4 *__restrict__ rec, const float4 *__restrict__ /* prjRec */, int totalTris,
                      int totalBins, int nframes)
{
    __shared__ StagedTri s_tri[kOccWarps][kOccChunk];
    __shared__ uint32_t s_rows[kOccWarps][kMaxLightN32][32];
    __shared__ uint32_t s_full[kOccWarps][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t(*rows)[32] = s_rows[warp];
    volatile uint32_t *sfull = s_full[warp];
    StagedTri *tris = s_tri[warp];
    unsigned long long tested = 0, nexam = 0, nchunks = 0, nrounds = 0;
    uint32_t nrows = 0, npart = 0;
    int nitems = *(volatile const int *)&ctr->itemCount;
    if (nitems > itemCapacity) nitems = itemCapacity;

    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(&ctr->itemCursor, 1);
        it = __shfl_sync(kFullWarp, it, 0);
        if (it >= nitems) break;
        const int4 item = items[it];
        const int bin = item.x, fi = item.z;
        if ((unsigned)bin >= (unsigned)totalBins || (unsigned)fi >= (unsigned)nframes) {
            if (lane == 0) atomicOr(&ctr->errorFlags, (int)ERR_INTERNAL);
            continue;
        }
        const FrameDesc &fr = frames[fi];
        const FrameState &st = states[fi];
        const int S = fr.W * fr.H;
        const int sLo = bss[bin] + item.y;
        const int sHi = min(sLo + kItemSamples, bse[bin]);
        const int tS = bts[bin];
        const int nT = bte[bin] - tS;

        if (nT <= 0) {
            // no triangle in this bin: shadow 0 -- or, in a later triangle pass,
            // the result of the earlier passes, left as it is
            if (!fr.accumulate) {
                for (int k = sLo + lane; k < sHi; k += 32) {
                    const int local = (int)sortedVals[k] - fr.sampleBase;
                    if ((unsigned)local < (unsigned)S) write_zero(fr, local);
                    else atomicOr(&ctr->errorFlags, (int)ERR_INTERNAL);
                }
            }
            continue;
        }

        const int N = fr.light.N;
        const uint32_t FULL = fr.light.full;
        const float nm1 = (float)(N - 1);
        const f3 xd = ld3(fr.light.xd), yd = ld3(fr.light.yd);
        const float esp = fr.esp;

        LaneSample smp;
        smp.Q = mk3(0.f, 0.f, 0.f);
        smp.L0Q = smp.Q;
        smp.spx = smp.spy = smp.spz = smp.spw = smp.spZ = 0.f;
        int local = 0;
        bool has = false;
        {
            const int k = sLo + lane;
            if (k < sHi) {
                local = (int)sortedVals[k] - fr.sampleBase;
                if ((unsigned)local >= (unsigned)S) {
                    atomicOr(&ctr->errorFlags, (int)ERR_INTERNAL);
                } else {
                    has = true;
                    load_sample(smp, fr, st, local);
                }
            }
        }
        uint32_t fr0 = FULL;
        if (has) fr0 = init_rows<uint32_t>(fr, local, grid_of<uint32_t>(fr), rows, lane);
        else
            for (int r = 0; r < N; ++r) rows[r][lane] = 0u;
        sfull[lane] = fr0;
        bool active = has && fr0 != FULL;
        for (int base = 0; base < nT && __any_sync(kFullWarp, active); base += kOccChunk) {
            const int m = min(kOccChunk, nT - base);
            __syncwarp();
            if (lane < m) {
                int tri = (int)(pairTri[tS + base + lane] & triMask);
                if ((unsigned)tri >= (unsigned)totalTris) {
                    atomicOr(&ctr->errorFlags, (int)ERR_INTERNAL);
                    tri = 0;
                }
                stage_triangle(tris[lane], rec, tri);
            }
            __syncwarp();
            // 1. cull: lane t keeps the samples passing triangle t
            uint32_t mine = 0u;
            for (int t = 0; t < m; ++t) {
                const float4 p0 = tris[t].p[0];
                const float minz = tris[t].p[1].x;
                const bool pass = active && p0.x <= smp.spx && p0.y <= smp.spy && smp.spz <= p0.z &&
                                  smp.spw <= p0.w && minz <= smp.spZ;
                const uint32_t b = __ballot_sync(kFullWarp, pass);
                if (lane == t) mine = b;
            }
            // 2. compute: pairs numbered triangle-major
            nexam += (unsigned long long)m * (unsigned)__popc(__ballot_sync(kFullWarp, active));
            ++nchunks;
            const int cnt = __popc(mine);
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(kFullWarp, incl, o);
                if (lane >= o) incl += y;
            }
            const int total = __shfl_sync(kFullWarp, incl, 31);
            const int excl = incl - cnt;
            for (int p0 = 0; p0 < total; p0 += 32) {
                ++nrounds;
                // (a) one pair per lane: edge coefficients and open rows
                const int p = p0 + lane;
                int t = 0;
#pragma unroll
                for (int w = 16; w >= 1; w >>= 1) {
                    const int e = __shfl_sync(kFullWarp, excl, t + w);
                    if (e <= p) t += w;
                }
                const uint32_t mt = __shfl_sync(kFullWarp, mine, t);
                const int kth = p - __shfl_sync(kFullWarp, excl, t);
                const bool valid = p < total;
                const int sl = valid ? nth_set_bit(mt, kth) : lane;
                const f3 Q = mk3(__shfl_sync(kFullWarp, smp.Q.x, sl), __shfl_sync(kFullWarp, smp.Q.y, sl),
                                 __shfl_sync(kFullWarp, smp.Q.z, sl));
                const f3 L0Q = mk3(__shfl_sync(kFullWarp, smp.L0Q.x, sl), __shfl_sync(kFullWarp, smp.L0Q.y, sl),
                                   __shfl_sync(kFullWarp, smp.L0Q.z, sl));
                PairEdges pe;
#pragma unroll
                for (int k = 0; k < 3; ++k) pe.A[k] = pe.B[k] = pe.C[k] = pe.Bn[k] = 0.0f;
                uint32_t vr = 0u;
                if (valid) {
                    const uint32_t fullRows = sfull[sl];
                    if (fullRows != FULL) {
                        ++tested;
                        vr = pair_setup(tris[t], Q, L0Q, xd, yd, esp, nm1, FULL, fullRows, pe, npart);
                    }
                }
                // (b) the (pair, row) units of this round, one per lane
                const int uc = __popc(vr);
                int uin = uc;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(kFullWarp, uin, o);
                    if (lane >= o) uin += y;
                }
                const int utotal = __shfl_sync(kFullWarp, uin, 31);
                const int uex = uin - uc;
                for (int u0 = 0; u0 < utotal; u0 += 32) {
                    const int u = u0 + lane;
                    int j = 0;
#pragma unroll
                    for (int w = 16; w >= 1; w >>= 1) {
                        const int e = __shfl_sync(kFullWarp, uex, j + w);
                        if (e <= u) j += w;
                    }
                    const uint32_t vj = __shfl_sync(kFullWarp, vr, j);
                    const int kk = u - __shfl_sync(kFullWarp, uex, j);
                    const int slj = __shfl_sync(kFullWarp, sl, j);
                    float A[3], B[3], C[3], Bn[3];
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        A[k] = __shfl_sync(kFullWarp, pe.A[k], j);
                        B[k] = __shfl_sync(kFullWarp, pe.B[k], j);
                        C[k] = __shfl_sync(kFullWarp, pe.C[k], j);
                        Bn[k] = __shfl_sync(kFullWarp, pe.Bn[k], j);
                    }
                    if (u < utotal) {
                        const int r = nth_set_bit(vj, kk);
                        ++nrows;
                        const float fr = (float)r;
                        uint32_t M = FULL;
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                            M &= row_mask_sel(__fadd_rn(__fmul_rn(A[k], fr), C[k]), Bn[k], B[k], FULL, npart);
                        if (M) {
                            const uint32_t old = atomicOr(&rows[r][slj], M);
                            if (old != FULL && (old | M) == FULL) atomicOr((uint32_t *)&sfull[slj], 1u << r);
                        }
                    }
                }
            }
            __syncwarp();
            active = active && sfull[lane] != FULL;
        }
        __syncwarp();
        if (has) write_result<uint32_t>(fr, local, grid_of<uint32_t>(fr), rows, lane);
    }
    unsigned long long t = tested, tr = nrows, tp = npart;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        t += __shfl_xor_sync(kFullWarp, t, o);
        tr += __shfl_xor_sync(kFullWarp, tr, o);
        tp += __shfl_xor_sync(kFullWarp, tp, o);
    }
    if (lane == 0 && t) {
        atomicAdd(&ctr->pairTests, t);
        atomicAdd(&ctr->rowsEvaluated, tr);
        atomicAdd(&ctr->partialMasks, tp);
    }
    if (lane == 0 && nchunks) {
        atomicAdd(&ctr->pairsExamined, nexam);
        atomicAdd(&ctr->chunks, nchunks);
        atomicAdd(&ctr->rounds, nrounds);
    }
}

}  // namespace fdzb
