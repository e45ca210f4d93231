// fdzb_pipeline.cu -- the B200 FDZB soft-shadow pipeline.
//
// Stage map (reference kernels in 4DZB/FDZB_Soft_Shadow/cuda/, "K/"):
//   k_init        clears per-launch bin state
//   k_reduce      k1+k2+k3+k4 fused: one pass over samples (pos+normal, 128-bit
//                 loads) and vertices computes the far-plane depth maxima and the
//                 sample / vertex rectangle bounds (K/Step2_1_*, K/Step2_2_*)
//   k_plan        light plane, far plane f, sub-constant, bin factor
//                 (K/Step2_3_defineFDbuffer.inl:5-111)
//   k_tri_setup   per-triangle cull + footprint AABB + 64-byte record
//                 (K/Step0_triangleSetup.inl:37-191)
//   k_sample_keys bin key per sample, back-facing/unbinned outputs, per-bin
//                 sample stats by warp-aggregated atomics (k6 + k9,
//                 K/Step3_bindSampleToBin.inl:5-104)
//   radix sort    sample pairs (k7) and triangle/bin pairs (k12), fdzb_sort.cuh
//   k_tri_pairs   count + decoupled look-back scan + pair write in one pass
//                 (k10 + exclusive_scan + k11, K/Step4_RasterizeTriangleToBin.inl)
//   k_items       per-bin work items for the occlusion kernel
//   k_occlusion   per-bin occlusion + popcount shading (k13,
//                 K/Step5_2_shadowCalPerSample.inl:37-231): a warp owns 32 samples
//                 of one bin; the bin's triangle records are staged into shared
//                 memory 32 at a time and every lane walks them against its own
//                 sample, OR-accumulating N-bit row masks.
#include "fdzb_device.cuh"
#include "fdzb_sort.cuh"
#include "fdzb_occlusion.cuh"

#include <mutex>
#include <string>


namespace fdzb {

// Vertex v of a frame's model: xyz from the caller's buffer, through the frame's
// model transform when it has one (the reference rewrites the buffer in place
// instead, K/moveModel.inl:14-28; both give the same floats).
__device__ __forceinline__ f3 load_vertex(const FrameDesc &fr, int v)
{
    const f3 q = ld3(fr.vtx + (size_t)v * fr.vstride);
    return fr.hasXform ? transform_point(fr.xform, q) : q;
}

// ---------------------------------------------------------------------------
// k_init: empty bin statistics (K/Step3_bindSampleToBin.inl:83-84) and cleared
// segment tables (K/binRaster.inl:39-40, 52-53).
// ---------------------------------------------------------------------------
__global__ void k_init(FrameState *states, int nframes, uint32_t *binStat, int32_t *bss,
                       int32_t *bse, int32_t *bts, int32_t *bte, int totalBins, uint32_t *epochWord)
{
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid == 0) *epochWord += 1u;  // launch number: look-back tags of this launch
    const int stride = gridDim.x * blockDim.x;
    const uint32_t neg = f2o(-kF32Max), pos = f2o(kF32Max);
    for (int b = gid; b < totalBins; b += stride) {
        uint4 s0 = make_uint4(neg, neg, neg, pos);
        uint4 s1 = make_uint4(pos, 0u, 0u, 0u);
        reinterpret_cast<uint4 *>(binStat)[2 * b] = s0;
        reinterpret_cast<uint4 *>(binStat)[2 * b + 1] = s1;
        bts[b] = kSegAbsent;   // segment bounds: lowered / raised by the sorts' last passes
        bte[b] = 0;
    }
    for (int b = gid; b <= totalBins; b += stride) {
        bss[b] = kSegAbsent;
        bse[b] = 0;
    }
    for (int f = gid; f < nframes; f += stride) {
        FrameState &s = states[f];
        s.acc[ACC_SMAXW] = f2o(-1.0f);  // thrust::reduce init value (K/Step2_1_*.inl:43)
        s.acc[ACC_TMAXW] = f2o(-1.0f);  // (K/Step2_2_*.inl:40)
        s.acc[ACC_S_MINU] = pos; s.acc[ACC_S_MINV] = pos; s.acc[ACC_S_MINW] = pos;
        s.acc[ACC_S_MAXA] = neg; s.acc[ACC_S_MAXB] = neg; s.acc[ACC_S_MAXW] = neg;
        s.acc[ACC_M_MINU] = pos; s.acc[ACC_M_MINV] = pos; s.acc[ACC_M_MINW] = pos;
        s.acc[ACC_M_MAXA] = neg; s.acc[ACC_M_MAXB] = neg; s.acc[ACC_M_MAXW] = neg;
        s.nFront = 0;
        s.state = 0;
        s.nValidTris = 0;
        s.nValidSamples = 0;
        s.quirkKeyRange = 0;
    }
}

// ---------------------------------------------------------------------------
// k_reduce: grid (x, frame, 2): z = 0 samples, z = 1 vertices.
// Sample part: k1 (max depth over non-background samples) and k3's bounds over
// front-facing samples.  The bound on rect.x + RF.x/w - sub is reduced before
// the subtraction (sub = RF/f needs f first): fl(x - sub) is monotone in x, so
// max_i fl(a_i - sub) == fl(max_i a_i - sub) exactly.
// Vertex part: k2 (max depth) and k4 (vertex rectangle bounds).
// ---------------------------------------------------------------------------
constexpr int kReduceThreads = 256;

__device__ __forceinline__ void acc_max(uint32_t &a, float v)
{
    if (!isnan(v)) a = max(a, f2o(v));
}
__device__ __forceinline__ void acc_min(uint32_t &a, float v)
{
    if (!isnan(v)) a = min(a, f2o(v));
}

__global__ void __launch_bounds__(kReduceThreads)
    k_reduce(const FrameDesc *__restrict__ frames, FrameState *states)
{
    const FrameDesc &fr = frames[blockIdx.y];
    FrameState &st = states[blockIdx.y];
    const float *M = fr.light.mat;
    const float RFx = fr.light.RF[0], RFy = fr.light.RF[1];
    __shared__ uint32_t s_acc[kReduceThreads / 32][8];
    __shared__ int s_cnt[kReduceThreads / 32];

    // slot layout in a[]: 0 max depth, 1 min u, 2 min v, 3 min w, 4 max a, 5 max b, 6 max w
    uint32_t a[7] = {0u, 0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    int cnt = 0;
    const int stride = gridDim.x * blockDim.x;
    if (blockIdx.z == 0) {
        const int S = fr.W * fr.H;
        const f3 ur = ld3(fr.light.ur), ul = ld3(fr.light.ul), dl = ld3(fr.light.dl),
                 dr = ld3(fr.light.dr);
        for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < S; p += stride) {
            const float4 P = __ldg(fr.pos + p);
            if (isnan(P.x)) continue;
            const f3 q = mk3(P.x, P.y, P.z);
            acc_max(a[0], light_depth(M, q));
            const float4 Nv = __ldg(fr.nrm + p);
            const f3 n = mk3(Nv.x, Nv.y, Nv.z);
            const bool back = dot3(sub3(ur, q), n) <= 0.0f && dot3(sub3(ul, q), n) <= 0.0f &&
                              dot3(sub3(dl, q), n) <= 0.0f && dot3(sub3(dr, q), n) <= 0.0f;
            if (back) continue;
            ++cnt;
            const f3 r = light_project(M, q);
            acc_min(a[1], r.x);
            acc_min(a[2], r.y);
            acc_min(a[3], r.z);
            acc_max(a[4], __fadd_rn(r.x, __fdiv_rn(RFx, r.z)));
            acc_max(a[5], __fadd_rn(r.y, __fdiv_rn(RFy, r.z)));
            acc_max(a[6], r.z);
        }
    } else {
        for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < fr.V; v += stride) {
            const f3 q = load_vertex(fr, v);
            acc_max(a[0], light_depth(M, q));
            const f3 r = light_project(M, q);
            acc_min(a[1], r.x);
            acc_min(a[2], r.y);
            acc_min(a[3], r.z);
            acc_max(a[4], __fadd_rn(r.x, __fdiv_rn(RFx, r.z)));
            acc_max(a[5], __fadd_rn(r.y, __fdiv_rn(RFy, r.z)));
            acc_max(a[6], r.z);
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t w[7];
    w[0] = __reduce_max_sync(kFullWarp, a[0]);
    w[1] = __reduce_min_sync(kFullWarp, a[1]);
    w[2] = __reduce_min_sync(kFullWarp, a[2]);
    w[3] = __reduce_min_sync(kFullWarp, a[3]);
    w[4] = __reduce_max_sync(kFullWarp, a[4]);
    w[5] = __reduce_max_sync(kFullWarp, a[5]);
    w[6] = __reduce_max_sync(kFullWarp, a[6]);
    const int c = __reduce_add_sync(kFullWarp, cnt);
    if (lane == 0) {
        for (int i = 0; i < 7; ++i) s_acc[warp][i] = w[i];
        s_cnt[warp] = c;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        const int i = threadIdx.x;
        if (i < 7) {
            uint32_t r = s_acc[0][i];
            const bool isMin = (i >= 1 && i <= 3);
            for (int k = 1; k < kReduceThreads / 32; ++k)
                r = isMin ? min(r, s_acc[k][i]) : max(r, s_acc[k][i]);
            const bool vert = blockIdx.z == 1;
            int slot;
            if (i == 0) slot = vert ? ACC_TMAXW : ACC_SMAXW;
            else slot = (vert ? ACC_M_MINU : ACC_S_MINU) + (i - 1);
            if (isMin) {
                if (r != 0xffffffffu) atomicMin(&st.acc[slot], r);
            } else {
                if (r != 0u) atomicMax(&st.acc[slot], r);
            }
        } else if (blockIdx.z == 0) {
            int t = 0;
            for (int k = 0; k < kReduceThreads / 32; ++k) t += s_cnt[k];
            if (t) atomicAdd(&st.nFront, t);
        }
    }
}

// ---------------------------------------------------------------------------
// k_plan: one thread per frame; host logic of lightPlaneParamCal
// (K/Step2_3_defineFDbuffer.inl:14-104) with the early exits as frame states.
// ---------------------------------------------------------------------------
__global__ void k_plan(const FrameDesc *__restrict__ frames, FrameState *states, int nframes)
{
    const int fi = blockIdx.x * blockDim.x + threadIdx.x;
    if (fi >= nframes) return;
    const FrameDesc &fr = frames[fi];
    FrameState &st = states[fi];
    const float smax = o2f(st.acc[ACC_SMAXW]);
    const float tmax = o2f(st.acc[ACC_TMAXW]);
    st.state = 0;
    if (smax < 0.0f || tmax < 0.0f) return;
    const float f = __fadd_rn(fmaxf(smax, tmax), 0.1f);
    const float subx = __fdiv_rn(fr.light.RF[0], f), suby = __fdiv_rn(fr.light.RF[1], f);
    st.f = f;
    st.subx = subx;
    st.suby = suby;
    st.state = 1;
    float s[6], m[6];
    s[0] = o2f(st.acc[ACC_S_MINU]);
    s[1] = o2f(st.acc[ACC_S_MINV]);
    s[2] = o2f(st.acc[ACC_S_MINW]);
    s[3] = st.nFront ? __fsub_rn(o2f(st.acc[ACC_S_MAXA]), subx) : -kF32Max;
    s[4] = st.nFront ? __fsub_rn(o2f(st.acc[ACC_S_MAXB]), suby) : -kF32Max;
    s[5] = o2f(st.acc[ACC_S_MAXW]);
    m[0] = o2f(st.acc[ACC_M_MINU]);
    m[1] = o2f(st.acc[ACC_M_MINV]);
    m[2] = o2f(st.acc[ACC_M_MINW]);
    m[3] = fr.V ? __fsub_rn(o2f(st.acc[ACC_M_MAXA]), subx) : -kF32Max;
    m[4] = fr.V ? __fsub_rn(o2f(st.acc[ACC_M_MAXB]), suby) : -kF32Max;
    m[5] = o2f(st.acc[ACC_M_MAXW]);
    for (int i = 0; i < 6; ++i) {
        st.sampleAabb[i] = s[i];
        st.modelAabb[i] = m[i];
    }
    if (st.nFront == 0) return;  // K/Step2_1_samplerRectangleAABB.inl:178-181
    if (m[0] > m[3] || m[1] > m[4] || s[0] > s[3] || s[1] > s[4]) return;
    st.Bx = fmaxf(s[0], m[0]);
    st.By = fmaxf(s[1], m[1]);
    st.Ex = fminf(s[3], m[3]);
    st.Ey = fminf(s[4], m[4]);
    st.Bz = m[2];
    st.Ez = s[5];
    if (st.Bx >= st.Ex || st.By >= st.Ey) return;
    st.fx = __fdiv_rn((float)fr.Wb, __fsub_rn(st.Ex, st.Bx));
    st.fy = __fdiv_rn((float)fr.Wb, __fsub_rn(st.Ey, st.By));
    st.state = 2;
}

// ---------------------------------------------------------------------------
// k_tri_setup: grid (x, frame).  Record layout (4 x float4 = 64 B):
//   q0 = (v0, minz) q1 = (v1, maxz) q2 = (v2, 1/w2) q3 = (aabb min x,y, aabb max x,y)
// and the vertices' projections for the occlusion stage's open-box test
// (2 x float4): (u0, v0, 1/w0, u1), (v1, 1/w1, u2, v2).
// Culled triangles keep the inverted AABB of the reference's triAABB buffer, so
// the pair counter's skip test rejects them exactly as K/Step4_*.inl:41 does.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    k_tri_setup(const FrameDesc *__restrict__ frames, FrameState *states, float4 *__restrict__ rec,
                float4 *__restrict__ prj, int *err)
{
    const FrameDesc &fr = frames[blockIdx.y];
    FrameState &st = states[blockIdx.y];
    if (st.state < 2) return;
    const float *M = fr.light.mat;
    const float RFx = fr.light.RF[0], RFy = fr.light.RF[1];
    const float subx = st.subx, suby = st.suby;
    const float Bx = st.Bx, By = st.By, Ex = st.Ex, Ey = st.Ey;
    const f3 ur = ld3(fr.light.ur), ul = ld3(fr.light.ul), dl = ld3(fr.light.dl),
             dr = ld3(fr.light.dr);
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < fr.T; base += stride) {
        const int t = base + lane;
        bool inLP = false;
        if (t < fr.T) {
            const int i0 = fr.idx[3 * (size_t)t], i1 = fr.idx[3 * (size_t)t + 1],
                      i2 = fr.idx[3 * (size_t)t + 2];
            float mnx = kF32Max, mny = kF32Max, mnz = kF32Max;
            float mxx = -kF32Max, mxy = -kF32Max, mxz = -kF32Max;
            float pu[3] = {0.f, 0.f, 0.f}, pv[3] = {0.f, 0.f, 0.f}, pw[3] = {0.f, 0.f, 0.f};
            f3 v0 = mk3(0.f, 0.f, 0.f), v1 = v0, v2 = v0;
            const bool okIdx = i0 >= 0 && i0 < fr.V && i1 >= 0 && i1 < fr.V && i2 >= 0 && i2 < fr.V;
            if (!okIdx) {
                atomicOr(err, (int)ERR_BAD_INPUT);
            } else {
                v0 = load_vertex(fr, i0);
                v1 = load_vertex(fr, i1);
                v2 = load_vertex(fr, i2);
                const f3 n = cross3(sub3(v0, v2), sub3(v1, v0));
                const bool culled =
                    fr.cull && dot3(n, sub3(ur, v0)) <= 0.0f && dot3(n, sub3(ur, v1)) <= 0.0f &&
                    dot3(n, sub3(ur, v2)) <= 0.0f && dot3(n, sub3(ul, v0)) <= 0.0f &&
                    dot3(n, sub3(ul, v1)) <= 0.0f && dot3(n, sub3(ul, v2)) <= 0.0f &&
                    dot3(n, sub3(dr, v0)) <= 0.0f && dot3(n, sub3(dr, v1)) <= 0.0f &&
                    dot3(n, sub3(dr, v2)) <= 0.0f && dot3(n, sub3(dl, v0)) <= 0.0f &&
                    dot3(n, sub3(dl, v1)) <= 0.0f && dot3(n, sub3(dl, v2)) <= 0.0f;
                if (!culled) {
                    const f3 vv[3] = {v0, v1, v2};
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const f3 r = light_project(M, vv[k]);
                        pu[k] = r.x;
                        pv[k] = r.y;
                        pw[k] = __frcp_rn(r.z);
                        mnx = fminf(mnx, r.x);
                        mny = fminf(mny, r.y);
                        mnz = fminf(mnz, r.z);
                        mxz = fmaxf(mxz, r.z);
                        mxx = fmaxf(mxx, __fsub_rn(__fadd_rn(r.x, __fdiv_rn(RFx, r.z)), subx));
                        mxy = fmaxf(mxy, __fsub_rn(__fadd_rn(r.y, __fdiv_rn(RFy, r.z)), suby));
                    }
                    inLP = !(mnx > Ex || mny > Ey || mxx < Bx || mxy < By);
                }
            }
            float4 *o = rec + 4 * (size_t)(fr.triBase + t);
            o[0] = make_float4(v0.x, v0.y, v0.z, mnz);
            o[1] = make_float4(v1.x, v1.y, v1.z, mxz);
            o[2] = make_float4(v2.x, v2.y, v2.z, pw[2]);
            o[3] = make_float4(mnx, mny, mxx, mxy);
            float4 *pp = prj + 2 * (size_t)(fr.triBase + t);
            pp[0] = make_float4(pu[0], pv[0], pw[0], pu[1]);
            pp[1] = make_float4(pv[1], pw[1], pu[2], pv[2]);
        }
        const unsigned b = __ballot_sync(kFullWarp, inLP);
        if (lane == 0 && b) atomicAdd(&st.nValidTris, __popc(b));
    }
}

// ---------------------------------------------------------------------------
// k_sample_keys: grid (x, frame).  k3's back-face/validity decision and
// rectangle, k6's key (K/Step3_bindSampleToBin.inl:29-57) and k9's per-bin
// statistics (max w, max rect.min x/y, min rect.max x/y; :61-104) by
// warp-aggregated atomics on order-preserving encodings.  Samples that get no
// bin receive their final output here: 1 (full mask) if back-facing, else 0.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    k_sample_keys(const FrameDesc *__restrict__ frames, FrameState *states, uint32_t *__restrict__ keys,
                  uint32_t *__restrict__ vals, uint32_t *binStat, int invalidKey)
{
    const FrameDesc &fr = frames[blockIdx.y];
    FrameState &st = states[blockIdx.y];
    const int state = st.state;
    const bool binning = state == 2 && st.nValidTris > 0;
    const float *M = fr.light.mat;
    const float RFx = fr.light.RF[0], RFy = fr.light.RF[1];
    const float subx = st.subx, suby = st.suby;
    const float Bx = st.Bx, By = st.By, Ex = st.Ex, Ey = st.Ey, fx = st.fx, fy = st.fy;
    const f3 ur = ld3(fr.light.ur), ul = ld3(fr.light.ul), dl = ld3(fr.light.dl),
             dr = ld3(fr.light.dr);
    const int S = fr.W * fr.H;
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    const int words = fr.maskWords;
    const int NN = fr.light.N * fr.light.NC;
    int nvalid = 0, nquirk = 0;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < S; base += stride) {
        const int p = base + lane;
        const bool in = p < S;
        bool valid = false, back = false;
        uint32_t key = (uint32_t)invalidKey;
        float w = 0.f, bx0 = 0.f, by0 = 0.f, ex0 = 0.f, ey0 = 0.f;
        if (in && state >= 1) {
            const float4 P = __ldg(fr.pos + p);
            if (!isnan(P.x)) {
                const float4 Nv = __ldg(fr.nrm + p);
                const f3 q = mk3(P.x, P.y, P.z), n = mk3(Nv.x, Nv.y, Nv.z);
                back = dot3(sub3(ur, q), n) <= 0.0f && dot3(sub3(ul, q), n) <= 0.0f &&
                       dot3(sub3(dl, q), n) <= 0.0f && dot3(sub3(dr, q), n) <= 0.0f;
                if (!back && binning) {
                    const f3 r = light_project(M, q);
                    bx0 = r.x;
                    by0 = r.y;
                    ex0 = __fsub_rn(__fadd_rn(r.x, __fdiv_rn(RFx, r.z)), subx);
                    ey0 = __fsub_rn(__fadd_rn(r.y, __fdiv_rn(RFy, r.z)), suby);
                    w = r.z;
                    if (!((bx0 > ex0 || by0 > ey0) || (bx0 < Bx || by0 < By || ex0 > Ex || ey0 > Ey))) {
                        // (e + b) / 2 of the reference: halving is exact, so the
                        // product by 0.5 is the same correctly rounded value
                        const float cx = __fmul_rn(__fadd_rn(ex0, bx0), 0.5f);
                        const float cy = __fmul_rn(__fadd_rn(ey0, by0), 0.5f);
                        const int bxi = __float2int_rz(floorf(__fmul_rn(__fsub_rn(cx, Bx), fx)));
                        const int byi = __float2int_rz(floorf(__fmul_rn(__fsub_rn(cy, By), fy)));
                        if (bxi >= 0 && bxi < fr.Wb && byi >= 0 && byi < fr.Wb) {
                            key = (uint32_t)(fr.binBase + ((byi << fr.log2Wb) | bxi));
                            valid = true;
                        } else {
                            ++nquirk;
                        }
                    }
                }
            }
        }
        if (in) {
            keys[fr.sampleBase + p] = key;
            vals[fr.sampleBase + p] = (uint32_t)(fr.sampleBase + p);
            if (!valid) {
                fr.shadow[p] = back ? 1.0f : 0.0f;
                if (fr.masks) {
                    uint32_t *mo = fr.masks + (size_t)p * words;
                    for (int wi = 0; wi < words; ++wi) {
                        uint32_t v = 0u;
                        if (back) {
                            const int rem = NN - 32 * wi;
                            v = rem >= 32 ? 0xffffffffu : ((1u << rem) - 1u);
                        }
                        mo[wi] = v;
                    }
                }
            }
        }
        // per-bin statistics, one atomic per distinct key per warp
        unsigned todo = __ballot_sync(kFullWarp, valid);
        nvalid += valid ? 1 : 0;
        while (todo) {
            const int leader = __ffs(todo) - 1;
            const uint32_t lk = __shfl_sync(kFullWarp, key, leader);
            const bool mine = valid && key == lk;
            const unsigned grp = __ballot_sync(kFullWarp, mine);
            const uint32_t mz = __reduce_max_sync(kFullWarp, mine ? f2o(w) : 0u);
            const uint32_t rx = __reduce_max_sync(kFullWarp, mine ? f2o(bx0) : 0u);
            const uint32_t ry = __reduce_max_sync(kFullWarp, mine ? f2o(by0) : 0u);
            const uint32_t rz = __reduce_min_sync(kFullWarp, mine ? f2o(ex0) : 0xffffffffu);
            const uint32_t rw = __reduce_min_sync(kFullWarp, mine ? f2o(ey0) : 0xffffffffu);
            if (lane == leader) {
                uint32_t *s = binStat + 8 * (size_t)lk;
                atomicMax(s + 0, mz);
                atomicMax(s + 1, rx);
                atomicMax(s + 2, ry);
                atomicMin(s + 3, rz);
                atomicMin(s + 4, rw);
            }
            todo &= ~grp;
        }
    }
    nvalid = __reduce_add_sync(kFullWarp, nvalid);
    nquirk = __reduce_add_sync(kFullWarp, nquirk);
    if (lane == 0) {
        if (nvalid) atomicAdd(&st.nValidSamples, nvalid);
        if (nquirk) atomicAdd(&st.quirkKeyRange, nquirk);
    }
}

// ---------------------------------------------------------------------------
// k_tri_pairs: persistent tiles of 256 triangles.  For each triangle, the
// candidate bins of its light-plane-clamped AABB are tested against the bin
// statistics (strict comparisons, K/Step4_RasterizeTriangleToBin.inl:74-103);
// the tile's pair count is scanned, the tile's global offset found by a
// decoupled look-back over previous tiles, and the (bin, triangle) pairs are
// written in triangle order, bins row-major -- the reference's layout
// (:184-202) with the counting predicate used for both passes.
// ---------------------------------------------------------------------------
constexpr int kTriThreads = 256;
constexpr int kTriTile = 64;   // triangles per pair-scan tile (launches of up to kTriSmallLaunch triangles)
constexpr int kTriSmallLaunch = 1 << 20;
// Look-back status word of a triangle tile: [63:32] launch epoch, [31:30] flag,
// [29:0] pair count (the pair capacity stays below 2^30).
constexpr unsigned long long kScanAgg = 1ull << 30;
constexpr unsigned long long kScanPrefix = 2ull << 30;
constexpr unsigned long long kScanMask = (1ull << 30) - 1ull;

struct TriBins {
    int cbx, cby, cex, cey;
    float bx, by, bz, ex, ey;
    bool any;
};

__device__ __forceinline__ TriBins tri_candidates(const float4 q0, const float4 q1, const float4 q3,
                                                  const FrameState &st, int Wb)
{
    TriBins r;
    r.any = false;
    float bx = q3.x, by = q3.y, bz = q0.w, ex = q3.z, ey = q3.w, ez = q1.w;
    if (bx > ex || by > ey || bz > ez || bx > st.Ex || by > st.Ey || ex < st.Bx || ey < st.By)
        return r;
    bx = fmaxf(bx, st.Bx);
    by = fmaxf(by, st.By);
    ex = fminf(ex, st.Ex);
    ey = fminf(ey, st.Ey);
    // float -> ushort conversions of the reference saturate to [0, 65535]
    const float fbx = fmaxf(floorf(__fmul_rn(__fsub_rn(bx, st.Bx), st.fx)), 0.0f);
    const float fby = fmaxf(floorf(__fmul_rn(__fsub_rn(by, st.By), st.fy)), 0.0f);
    const float fex = fminf(ceilf(__fmul_rn(__fsub_rn(ex, st.Bx), st.fx)), (float)Wb);
    const float fey = fminf(ceilf(__fmul_rn(__fsub_rn(ey, st.By), st.fy)), (float)Wb);
    r.cbx = (int)__float2uint_rz(fminf(fbx, 65535.0f));
    r.cby = (int)__float2uint_rz(fminf(fby, 65535.0f));
    r.cex = (int)__float2uint_rz(fmaxf(fex, 0.0f));
    r.cey = (int)__float2uint_rz(fmaxf(fey, 0.0f));
    r.bx = bx; r.by = by; r.bz = bz; r.ex = ex; r.ey = ey;
    r.any = true;
    return r;
}

// A candidate bin whose statistics (max sample depth, the samples' rectangle
// extremes; words 0-4 of the bin record) the triangle's footprint can reach:
// the strict bin filter of K/Step4_RasterizeTriangleToBin.inl:94,193.
__device__ __forceinline__ bool stat_accepts(uint4 s, uint32_t s4, const TriBins &c)
{
    const float maxz = o2f(s.x), Rx = o2f(s.y), Ry = o2f(s.z), Rz = o2f(s.w), Rw = o2f(s4);
    return maxz >= c.bz && c.bx < Rx && c.by < Ry && Rz < c.ex && Rw < c.ey;
}

// Coverage-order bucket of a triangle (the key of the triangle sort): the triangle's
// angular size seen from below, world area / (f - minz)^2 with f - minz the
// light-depth distance from the far plane (about the receivers' depth) to the
// triangle's vertex nearest the light, as a log-scale bucket; the largest
// come first.  A sample's mask is the OR over its bin's triangles, so the order
// changes only how soon its light rows fill (the early-out), never the result.
__device__ __forceinline__ uint32_t coverage_bucket(const float4 *__restrict__ rec, int g, float f, int depthBits)
{
    if (depthBits <= 0) return 0u;   // reference order: the reference's (bin, triangle) order
    const float4 r0 = __ldg(&rec[4 * (size_t)g]), r1 = __ldg(&rec[4 * (size_t)g + 1]),
                 r2 = __ldg(&rec[4 * (size_t)g + 2]);
    const float ax = r1.x - r0.x, ay = r1.y - r0.y, az = r1.z - r0.z;
    const float bx = r2.x - r0.x, by = r2.y - r0.y, bz = r2.z - r0.z;
    const float cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
    const float area2 = fmaxf(sqrtf(cx * cx + cy * cy + cz * cz), 1e-30f);
    const float d = fmaxf(f - r0.w, 1e-6f);   // r0.w: the triangle's least light depth
    const float nb = (float)(1 << depthBits);
    const float q = -log2f(area2 / (d * d)) * (nb / 40.0f) + 0.5f * nb;
    return (uint32_t)(int)fminf(fmaxf(q, 0.0f), nb - 1.0f);
}

// k_tri_order: the coverage order's sort input, (bucket, triangle id) for every
// triangle; triangles of frames without a light plane go last (they emit no
// pairs either way).
__global__ void k_tri_order(const FrameState *__restrict__ states, const int *__restrict__ triBases, int nframes,
                            int totalTris, const float4 *__restrict__ rec, int depthBits,
                            uint32_t *__restrict__ keys, uint32_t *__restrict__ vals)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < totalTris; g += gridDim.x * blockDim.x) {
        const FrameState &st = states[frame_of(triBases, nframes, g)];
        keys[g] = (st.state == 2 && st.nValidTris > 0) ? coverage_bucket(rec, g, st.f, depthBits)
                                                       : (1u << depthBits) - 1u;
        vals[g] = (uint32_t)g;
    }
}

// Candidate bins of a triangle, swept by a warp 32 at a time in row-major
// order; returns the number accepted and, with write, writes the accepted
// (bin, triangle) pairs from position `pos` on, in order: as (key = bin,
// value = triangle), or, with triBits > 0, as the one word
// bin << triBits | triangle.
__device__ __forceinline__ int sweep_bins(const uint32_t *__restrict__ binStat, const TriBins &c, int bb, int l2,
                                          int lane, uint32_t *__restrict__ pkeys, uint32_t *__restrict__ pvals,
                                          unsigned long long pos, int capacity, int g, bool write, int triBits)
{
    const int w = c.cex - c.cbx, h = c.cey - c.cby;
    if (w <= 0 || h <= 0) return 0;
    const int n = w * h;
    int total = 0;
    // lane's slot li = base + lane; (j, i) kept incrementally
    int j = c.cby + lane / w, i = c.cbx + lane % w;
    const int stepJ = 32 / w, stepI = 32 % w;
    // the bin statistics of the lane's next slot are loaded one round ahead,
    // so that their latency overlaps the current round
    const uint4 *stat4 = reinterpret_cast<const uint4 *>(binStat);
    uint4 sc = make_uint4(0u, 0u, 0u, 0u);
    uint32_t sc4 = 0u;
    if (lane < n) {
        const int g0 = bb + ((j << l2) | i);
        sc = __ldg(stat4 + 2 * (size_t)g0);
        sc4 = __ldg(binStat + 8 * (size_t)g0 + 4);
    }
    for (int base = 0; base < n; base += 32) {
        const int li = base + lane;
        bool ok = false;
        int gb = 0;
        int jn = j + stepJ, inx = i + stepI;
        if (inx >= c.cex) {
            inx -= w;
            ++jn;
        }
        uint4 sn = make_uint4(0u, 0u, 0u, 0u);
        uint32_t sn4 = 0u;
        if (li + 32 < n) {
            const int gn = bb + ((jn << l2) | inx);
            sn = __ldg(stat4 + 2 * (size_t)gn);
            sn4 = __ldg(binStat + 8 * (size_t)gn + 4);
        }
        if (li < n) {
            gb = bb + ((j << l2) | i);
            ok = stat_accepts(sc, sc4, c);
        }
        const unsigned m = __ballot_sync(kFullWarp, ok);
        if (write && ok) {
            const unsigned long long p = pos + (unsigned long long)total + (unsigned)__popc(m & lanemask_lt());
            if (p < (unsigned long long)capacity) {
                if (triBits) {
                    pkeys[p] = ((uint32_t)gb << triBits) | (uint32_t)g;
                } else {
                    pkeys[p] = (uint32_t)gb;
                    pvals[p] = (uint32_t)g;
                }
            }
        }
        total += __popc(m);
        j = jn;
        i = inx;
        sc = sn;
        sc4 = sn4;
    }
    return total;
}

// k_tri_pairs: persistent tiles of TILE triangles; a warp takes the
// tile's triangles in turn (warp w: triangles w, w + 8, ...) and sweeps each
// one's candidate bins with its 32 lanes.  Count pass, block scan of the
// per-triangle counts, decoupled look-back over tiles for the tile's global
// offset, then the write pass in the same order: pairs come out in triangle
// order, bins row-major -- the reference's layout.  With `order` (the coverage
// order) the i-th triangle processed is order[i] instead of i.
// 4 blocks of 256 threads per SM (64 registers; 70 without the bound, which
// leaves 3): with the prefetch in the sweep, HD pairs 0.325 -> 0.272 ms.
template <int TILE>
__global__ void __launch_bounds__(kTriThreads, 4)
    k_tri_pairs(const FrameDesc *__restrict__ frames, const FrameState *__restrict__ states,
                const int *__restrict__ triBases, int nframes, int totalTris,
                const float4 *__restrict__ rec, const uint32_t *__restrict__ binStat,
                int32_t *__restrict__ triCount, unsigned long long *scanStatus, const uint32_t *epochWord,
                uint32_t *__restrict__ pkeys, uint32_t *__restrict__ pvals, int capacity,
                const uint32_t *__restrict__ order, int triBits, Counters *ctr)
{
    constexpr int WARPS = kTriThreads / 32;
    constexpr int TPW = TILE / WARPS;   // triangles per warp and tile
    static_assert(TILE % WARPS == 0 && TPW <= 32 && TILE <= kTriThreads, "tile of 8..256 triangles");
    __shared__ int s_tile;
    __shared__ int s_cnt[TILE];
    __shared__ unsigned long long s_wsum[WARPS];
    __shared__ unsigned long long s_excl;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ntiles = (totalTris + TILE - 1) / TILE;
    const uint32_t epoch = *epochWord;
    for (;;) {
        __syncthreads();
        if (tid == 0) s_tile = atomicAdd(&ctr->triTileCounter, 1);
        __syncthreads();
        const int tile = s_tile;
        if (tile >= ntiles) break;
        const int t0 = tile * TILE;
        // Each of the first TPW lanes prepares one of the warp's triangles of
        // the tile (k = warp + 8 lane): order, record and candidate bins are
        // loaded for all at once, and the sweeps take them from the owning lane.
        TriBins myC;
        myC.any = false;
        myC.cbx = myC.cby = myC.cex = myC.cey = 0;
        myC.bx = myC.by = myC.bz = myC.ex = myC.ey = 0.0f;
        int myG = -1, myBB = 0, myL2 = 0;
        if (lane < TPW) {
            const int i = t0 + warp + WARPS * lane;
            const int g = (order && i < totalTris) ? (int)order[i] : i;
            if (i < totalTris && (unsigned)g < (unsigned)totalTris) {
                myG = g;
                const int fi = frame_of(triBases, nframes, g);
                const FrameState &st = states[fi];
                if (st.state == 2 && st.nValidTris > 0) {
                    const float4 q0 = __ldg(rec + 4 * (size_t)g), q1 = __ldg(rec + 4 * (size_t)g + 1),
                                 q3 = __ldg(rec + 4 * (size_t)g + 3);
                    myC = tri_candidates(q0, q1, q3, st, frames[fi].Wb);
                    myBB = frames[fi].binBase;
                    myL2 = frames[fi].log2Wb;
                }
            }
        }
        auto take = [&](int j, TriBins &c, int &g, int &bb, int &l2) {
            c.cbx = __shfl_sync(kFullWarp, myC.cbx, j);
            c.cby = __shfl_sync(kFullWarp, myC.cby, j);
            c.cex = __shfl_sync(kFullWarp, myC.cex, j);
            c.cey = __shfl_sync(kFullWarp, myC.cey, j);
            c.bx = __shfl_sync(kFullWarp, myC.bx, j);
            c.by = __shfl_sync(kFullWarp, myC.by, j);
            c.bz = __shfl_sync(kFullWarp, myC.bz, j);
            c.ex = __shfl_sync(kFullWarp, myC.ex, j);
            c.ey = __shfl_sync(kFullWarp, myC.ey, j);
            c.any = __shfl_sync(kFullWarp, (int)myC.any, j) != 0;
            g = __shfl_sync(kFullWarp, myG, j);
            bb = __shfl_sync(kFullWarp, myBB, j);
            l2 = __shfl_sync(kFullWarp, myL2, j);
        };
        // count pass: warp per triangle
        for (int j = 0; j < TPW; ++j) {
            const int k = warp + WARPS * j;
            TriBins c;
            int g, bb, l2;
            take(j, c, g, bb, l2);
            int cnt = 0;
            if (g >= 0) {
                if (c.any) cnt = sweep_bins(binStat, c, bb, l2, lane, pkeys, pvals, 0, capacity, g, false, triBits);
                if (lane == 0) triCount[g] = cnt;
            }
            if (lane == 0) s_cnt[k] = cnt;
        }
        __syncthreads();
        // block inclusive scan of the per-triangle counts (thread tid holds triangle tid)
        const int cnt = tid < TILE ? s_cnt[tid] : 0;
        unsigned long long x = (unsigned long long)cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long y = __shfl_up_sync(kFullWarp, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_wsum[warp] = x;
        __syncthreads();
        unsigned long long wbase = 0, total = 0;
        for (int w = 0; w < WARPS; ++w) {
            if (w < warp) wbase += s_wsum[w];
            total += s_wsum[w];
        }
        const unsigned long long mine_excl = wbase + x - (unsigned long long)cnt;
        __syncthreads();
        if (tid < TILE)
            s_cnt[tid] = (int)min(mine_excl, (unsigned long long)0x7fffffff);   // now: exclusive offset in the tile
        if (tid == 0) {
            unsigned long long excl = 0;
            unsigned long long *my = scanStatus + tile;
            const unsigned long long ep = (unsigned long long)epoch << 32;
            const unsigned long long tot = total > kScanMask ? kScanMask : total;
            if (tile == 0) {
                st_volatile_u64(my, ep | kScanPrefix | tot);
            } else {
                st_volatile_u64(my, ep | kScanAgg | tot);
                int t = tile - 1;
                unsigned spins = 0;
                while (t >= 0) {
                    const unsigned long long s = ld_volatile_u64(scanStatus + t);
                    const unsigned long long flag = ((s >> 32) == epoch) ? (s & 0xC0000000ull) : 0ull;
                    if (flag == 0) {
                        if (++spins > kSpinLimit) {
                            atomicOr(&ctr->errorFlags, (int)ERR_LOOKBACK_TIMEOUT);
                            break;
                        }
                        continue;
                    }
                    excl += s & kScanMask;
                    if (flag == kScanPrefix) break;
                    --t;
                }
                const unsigned long long inc = excl + total > kScanMask ? kScanMask : excl + total;
                st_volatile_u64(my, ep | kScanPrefix | inc);
            }
            s_excl = excl;
            if (tile == ntiles - 1) {
                const unsigned long long all = excl + total;
                ctr->pairCount = (int)(all > 0x7fffffffull ? 0x7fffffffull : all);
                if (all > (unsigned long long)capacity) ctr->pairOverflow = 1;
            }
        }
        __syncthreads();
        // write pass, same order
        const unsigned long long tileBase = s_excl;
        for (int j = 0; j < TPW; ++j) {
            const int k = warp + WARPS * j;
            TriBins c;
            int g, bb, l2;
            take(j, c, g, bb, l2);
            if (g < 0 || !c.any) continue;
            sweep_bins(binStat, c, bb, l2, lane, pkeys, pvals, tileBase + (unsigned long long)s_cnt[k], capacity, g,
                       true, triBits);
        }
    }
}

// ---------------------------------------------------------------------------
// k_move_model: FD::moveModel (K/moveModel.inl:6-30): xyz <- M * (xyz, 1) in
// place, each component summed left to right.
// ---------------------------------------------------------------------------
static int grid_for_host(long long n, int threads, int cap)
{
    long long g = (n + threads - 1) / threads;
    return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

struct Mat16 {
    float m[16];
};

__global__ void k_move_model(float *vtx, int vstride, int V, Mat16 M)
{
    const float *m = M.m;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        float *p = vtx + (size_t)v * vstride;
        const f3 r = transform_point(m, mk3(p[0], p[1], p[2]));
        p[0] = r.x;
        p[1] = r.y;
        p[2] = r.z;
    }
}

cudaError_t run_move_model(float *vtx, int vstride, int V, const float m[16], cudaStream_t s)
{
    Mat16 M;
    for (int i = 0; i < 16; ++i) M.m[i] = m[i];
    if (V <= 0) return cudaSuccess;
    k_move_model<<<grid_for_host(V, 256, 148 * 8), 256, 0, s>>>(vtx, vstride, V, M);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Host driver.
// ---------------------------------------------------------------------------
static_assert(kSortTileHost == kSortTile, "sort tile mismatch");
static_assert(kTriTileHost == kTriTile, "pair-scan tile mismatch");

int sort_passes_for(long long keyRangeExclusive)
{
    int bits = 0;
    while (bits < 32 && (1ll << bits) < keyRangeExclusive) ++bits;
    if (bits == 0) bits = 1;
    return (bits + 7) / 8;
}

static int grid_for(long long n, int threads, int cap)
{
    long long g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

// Keys-only passes (packed pairs): 64 registers, so 4 blocks of 256 threads
// per SM (pair sort at HD 0.353 -> 0.343 ms; 5 blocks spill, 6144-key tiles
// spill and gain nothing).
#ifndef FDZB_SORTK_ITEMS
#define FDZB_SORTK_ITEMS 16
#endif
#ifndef FDZB_SORTK_MINBLOCKS
#define FDZB_SORTK_MINBLOCKS 4
#endif
constexpr int kKeysItems = FDZB_SORTK_ITEMS, kKeysMinBlocks = FDZB_SORTK_MINBLOCKS;
constexpr int kKeysTile = kSortThreads * kKeysItems;
static_assert(kKeysTile >= kSortTile, "the look-back status array is sized for tiles of kSortTile keys");

// Sorts (kA, vA) with kB/vB as ping-pong buffers; `slot` selects the histogram
// and ticket block (0 samples, 1 pairs, 2 triangles).  Pass p uses tag
// 16*launch + 4*slot + p and the key's bits [shift0 + 8p, shift0 + 8p + 8).
// vA == nullptr: keys alone.  With segStart/segEnd the last pass also writes
// the bounds of the segments key >> segShift (nslots of them; K/binRaster.inl:5-33).
static void run_sort(const DeviceBuffers &b, int slot, uint32_t *kA, uint32_t *vA, uint32_t *kB,
                     uint32_t *vB, const int *n_dev, int n_static, int cap, int passes, int sm,
                     cudaStream_t s, int shift0 = 0, int32_t *segStart = nullptr, int32_t *segEnd = nullptr,
                     int segShift = 0, uint32_t nslots = 0)
{
    uint32_t *hist = b.sortHist + slot * 4 * kRadix;
    k_radix_hist<<<grid_for(cap, kSortThreads, sm * 4), kSortThreads, 0, s>>>(kA, n_dev, n_static,
                                                                              cap, passes, shift0, hist);
    uint32_t *ki = kA, *vi = vA, *ko = kB, *vo = vB;
    const long long tiles = ((long long)cap + kSortTile - 1) / kSortTile;
    const int passGrid = grid_for(tiles * kSortThreads, kSortThreads, sm * 4);
    const long long keysTiles = ((long long)cap + kKeysTile - 1) / kKeysTile;
    const int keysGrid = grid_for(keysTiles * kSortThreads, kSortThreads, sm * kKeysMinBlocks);
    for (int p = 0; p < passes; ++p) {
        const bool seg = segStart && p == passes - 1;
#define FDZB_PASS_ARGS(VI, VO)                                                                               \
    ki, VI, ko, VO, n_dev, n_static, cap, shift0 + 8 * p, hist + p * kRadix, b.sortStatus, b.epochWord,      \
        (uint32_t)(slot * 4 + p), b.counters->sortTileCounter + slot * 4 + p, &b.counters->errorFlags
        if (vA && seg)
            k_radix_pass<true, kSortItems, FDZB_SORT_MINBLOCKS, true><<<passGrid, kSortThreads, 0, s>>>(
                FDZB_PASS_ARGS(vi, vo), segStart, segEnd, segShift, nslots);
        else if (vA)
            k_radix_pass<true><<<passGrid, kSortThreads, 0, s>>>(FDZB_PASS_ARGS(vi, vo));
        else if (seg)
            k_radix_pass<false, kKeysItems, kKeysMinBlocks, true><<<keysGrid, kSortThreads, 0, s>>>(
                FDZB_PASS_ARGS(nullptr, nullptr), segStart, segEnd, segShift, nslots);
        else
            k_radix_pass<false, kKeysItems, kKeysMinBlocks><<<keysGrid, kSortThreads, 0, s>>>(
                FDZB_PASS_ARGS(nullptr, nullptr));
#undef FDZB_PASS_ARGS
        uint32_t *t = ki;
        ki = ko;
        ko = t;
        t = vi;
        vi = vo;
        vo = t;
    }
}


static int g_smCount = 0;

static int sm_count()
{
    if (g_smCount == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_smCount, cudaDevAttrMultiProcessorCount, dev);
        if (g_smCount <= 0) g_smCount = 148;
    }
    return g_smCount;
}

cudaError_t run_pipeline(const DeviceBuffers &b, int maxS, int maxT, int maxV, cudaStream_t s,
                         cudaEvent_t *ev, int *launches)
{
    const int sm = sm_count();
    const int nf = b.nframes;
    int nl = 0;
    if (ev) cudaEventRecord(ev[STAGE_SETUP], s);
    // (a) samples, vertices, triangles
    k_init<<<grid_for(b.totalBins + 1, 256, sm * 8), 256, 0, s>>>(
        b.states, nf, b.binStat, b.binSampleStart, b.binSampleEnd, b.binTriStart, b.binTriEnd, b.totalBins,
        b.epochWord);
    {
        const int gx = grid_for(maxS > maxV ? maxS : maxV, kReduceThreads, sm * 4);
        k_reduce<<<dim3(gx, nf, 2), kReduceThreads, 0, s>>>(b.frames, b.states);
    }
    k_plan<<<(nf + 63) / 64, 64, 0, s>>>(b.frames, b.states, nf);
    k_tri_setup<<<dim3(grid_for(maxT, 256, sm * 8), nf), 256, 0, s>>>(b.frames, b.states, b.triRec,
                                                                      b.triPrj, &b.counters->errorFlags);
    k_sample_keys<<<dim3(grid_for(maxS, 256, sm * 8), nf), 256, 0, s>>>(
        b.frames, b.states, b.keysA, b.valsA, b.binStat, b.totalBins);
    nl += 5;
    if (b.dbgKeys) {
        cudaMemcpyAsync(b.dbgKeys, b.keysA, 4ull * b.totalSamples, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(b.dbgVals, b.valsA, 4ull * b.totalSamples, cudaMemcpyDeviceToDevice, s);
    }
    // (b) sample sort and segments
    if (ev) cudaEventRecord(ev[STAGE_SAMPLE_SORT], s);
    run_sort(b, 0, b.keysA, b.valsA, b.keysB, b.valsB, nullptr, b.totalSamples, b.totalSamples,
             b.samplePasses, sm, s, 0, b.binSampleStart, b.binSampleEnd, 0, (uint32_t)b.totalBins + 1u);
    uint32_t *sv = (b.samplePasses & 1) ? b.valsB : b.valsA;
    nl += 1 + b.samplePasses;
    // (a) triangle/bin pairs, in the coverage order when one is asked for
    if (ev) cudaEventRecord(ev[STAGE_TRI_PAIRS], s);
    const uint32_t *order = nullptr;
    if (b.depthBits > 0 && b.totalTris > 0) {
        k_tri_order<<<grid_for(b.totalTris, 256, sm * 8), 256, 0, s>>>(b.states, b.triBases, nf, b.totalTris,
                                                                     b.triRec, b.depthBits, b.tkeysA, b.tvalsA);
        run_sort(b, 2, b.tkeysA, b.tvalsA, b.tkeysB, b.tvalsB, nullptr, b.totalTris, b.totalTris, b.triPasses,
                 sm, s);
        order = (b.triPasses & 1) ? b.tvalsB : b.tvalsA;
        nl += 2 + b.triPasses;
    }
    {
        // tiles of 64 triangles, 8 a warp, up to a million triangles: a frame
        // of few triangles still spreads over the SMs (2k triangles: pairs
        // 0.159 -> 0.074 ms against tiles of 256; HD: 0.305 -> 0.277 ms);
        // above, tiles of 256 (64 frames, 8.9M triangles: 7.1 ms against 8.4
        // ms with tiles of 64).  Up to 8 blocks per SM: the sweeps wait on
        // bin-statistics loads, so more resident warps hide more of that latency.
        const bool small = b.totalTris <= kTriSmallLaunch;
        const int tile = small ? kTriTile : 256;
        const int tiles = (b.totalTris + tile - 1) / tile;
        const int grid = tiles < sm * 8 ? (tiles > 0 ? tiles : 1) : sm * 8;
        if (small)
            k_tri_pairs<kTriTile><<<grid, kTriThreads, 0, s>>>(b.frames, b.states, b.triBases, nf, b.totalTris,
                                                               b.triRec, b.binStat, b.triCount, b.triScanStatus,
                                                               b.epochWord, b.pkeysA, b.pvalsA, b.pairCapacity,
                                                               order, b.pairTriBits, b.counters);
        else
            k_tri_pairs<256><<<grid, kTriThreads, 0, s>>>(b.frames, b.states, b.triBases, nf, b.totalTris,
                                                          b.triRec, b.binStat, b.triCount, b.triScanStatus,
                                                          b.epochWord, b.pkeysA, b.pvalsA, b.pairCapacity,
                                                          order, b.pairTriBits, b.counters);
        nl += 1;
    }
    if (b.dbgPKeys) {
        cudaMemcpyAsync(b.dbgPKeys, b.pkeysA, 4ull * b.pairCapacity, cudaMemcpyDeviceToDevice, s);
        if (!b.pairTriBits)
            cudaMemcpyAsync(b.dbgPVals, b.pvalsA, 4ull * b.pairCapacity, cudaMemcpyDeviceToDevice, s);
    }
    // (b) pair sort and segments
    if (ev) cudaEventRecord(ev[STAGE_PAIR_SORT], s);
    // packed pairs (pairTriBits > 0): the keys alone are sorted on their bin
    // bits, and the sorted keys are the triangle lists
    const bool packed = b.pairTriBits > 0;
    run_sort(b, 1, b.pkeysA, packed ? nullptr : b.pvalsA, b.pkeysB, packed ? nullptr : b.pvalsB,
             &b.counters->pairCount, 0, b.pairCapacity, b.pairPasses, sm, s, b.pairTriBits, b.binTriStart,
             b.binTriEnd, b.pairTriBits, (uint32_t)b.totalBins);
    uint32_t *pk = (b.pairPasses & 1) ? b.pkeysB : b.pkeysA;
    uint32_t *pv = packed ? pk : ((b.pairPasses & 1) ? b.pvalsB : b.pvalsA);
    const uint32_t triMask = packed ? (1u << b.pairTriBits) - 1u : 0xFFFFFFFFu;
    nl += 1 + b.pairPasses;
    // (c) + (d) occlusion and shading
    if (ev) cudaEventRecord(ev[STAGE_OCCLUSION], s);
    k_items<<<grid_for(b.totalBins, 256, sm * 8), 256, 0, s>>>(
        b.frames, b.binSampleStart, b.binSampleEnd, b.binTriStart, b.binTriEnd, b.binBases, nf, b.totalBins,
        b.items, b.itemCapacity, b.counters);
    // 64-bit row words when some frame's grid exceeds 32 rows or columns; the
    // lane-per-pair schedule only runs square 32-bit grids without the depth
    // plane (the host falls back to lane per sample otherwise)
    typedef RowWord<u64> W64;
    const int g32 = sm * FDZB_OCC_MINBLOCKS, g64 = sm * W64::kMinBlocks, t64 = W64::kWarps * 32;
#define FDZB_OCC_ARGS                                                                                        \
    b.frames, b.states, b.items, b.itemCapacity, b.counters, sv, b.binSampleStart, b.binSampleEnd, b.binTriStart, \
        b.binTriEnd, pv, triMask, b.triRec, b.triPrj, b.totalTris, b.totalBins, nf
    // b.openBox: the open-box cull's instantiation (edge-function masks only);
    // b.countWork: the instantiation that accumulates the work counters
#define FDZB_OCC(RC, RT, DP, BX, G, T)                                                                        \
    do {                                                                                                   \
        if (b.countWork) k_occlusion<RC, RT, DP, BX, 1><<<G, T, 0, s>>>(FDZB_OCC_ARGS);                     \
        else k_occlusion<RC, RT, DP, BX, 0><<<G, T, 0, s>>>(FDZB_OCC_ARGS);                                 \
    } while (0)
    // grids of at most 16 rows: the lanes' masks in 16-row shared arrays
#define FDZB_OCC16(DP, BX)                                                                                    \
    do {                                                                                                   \
        if (b.countWork) k_occlusion<0, uint32_t, DP, BX, 1, 16><<<g32, kOccThreads, 0, s>>>(FDZB_OCC_ARGS); \
        else k_occlusion<0, uint32_t, DP, BX, 0, 16><<<g32, kOccThreads, 0, s>>>(FDZB_OCC_ARGS);             \
    } while (0)
    if (b.wide) {
        if (b.rayCast) FDZB_OCC(1, u64, 0, 0, g64, t64);
        else if (b.depthPlane && b.openBox) FDZB_OCC(0, u64, 1, 1, g64, t64);
        else if (b.depthPlane) FDZB_OCC(0, u64, 1, 0, g64, t64);
        else if (b.openBox) FDZB_OCC(0, u64, 0, 1, g64, t64);
        else FDZB_OCC(0, u64, 0, 0, g64, t64);
    } else if (b.rayCast) {
        FDZB_OCC(1, uint32_t, 0, 0, g32, kOccThreads);
    } else if (b.occVariant == 1) {
        k_occlusion_pairs<<<sm * FDZB_OCC2_MINBLOCKS, kOccThreads, 0, s>>>(FDZB_OCC_ARGS);
    } else if (b.depthPlane) {
        if (b.openBox && b.rows16) FDZB_OCC16(1, 1);
        else if (b.openBox) FDZB_OCC(0, uint32_t, 1, 1, g32, kOccThreads);
        else if (b.rows16) FDZB_OCC16(1, 0);
        else FDZB_OCC(0, uint32_t, 1, 0, g32, kOccThreads);
    } else if (b.openBox) {
        if (b.rows16) FDZB_OCC16(0, 1);
        else FDZB_OCC(0, uint32_t, 0, 1, g32, kOccThreads);
    } else {
        if (b.rows16) FDZB_OCC16(0, 0);
        else FDZB_OCC(0, uint32_t, 0, 0, g32, kOccThreads);
    }
#undef FDZB_OCC
#undef FDZB_OCC16
#undef FDZB_OCC_ARGS
    nl += 2;
    if (ev) cudaEventRecord(ev[STAGE_COUNT], s);
    if (launches) *launches = nl;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Issue-rate probe for the roofline of the occlusion kernel: 8 independent
// FP32 add chains per thread, enough warps per SM to hide the add latency.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_alu_probe(float *out, int iters, float step)
{
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = (float)(threadIdx.x + k) * 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = __fadd_rn(a[k], step);
    }
    float r = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) r = __fadd_rn(r, a[k]);
    if (r == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = r;  // keeps the chains live
}

cudaError_t measure_alu_rate(double *rate)
{
    const int sm = sm_count();
    float *out = nullptr;
    cudaError_t e = cudaMalloc(&out, 4);
    if (e != cudaSuccess) return e;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = sm * 8, threads = 256, iters = 4096;
    k_alu_probe<<<blocks, threads>>>(out, 64, 1.0f);  // warm-up
    cudaEventRecord(a);
    k_alu_probe<<<blocks, threads>>>(out, iters, 1.0f);
    cudaEventRecord(b);
    e = cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    if (e == cudaSuccess) e = cudaGetLastError();
    *rate = ms > 0 ? (double)blocks * threads * iters * 8.0 / (ms * 1e-3) : 0.0;
    return e;
}

// ---------------------------------------------------------------------------
// Self-check of the occlusion rows' quotient.  k_check_reciprocal enumerates
// every float b with |b| in [2^-100, 2^40) (both signs) and compares
// rcp_nearest(b) with __frcp_rn(b).  k_check_division compares
// div_by_rcp(a, b, rcp_nearest(b)) with the IEEE division __fdiv_rn, over
// the operand ranges the pair test admits to it.
// Trial t draws (from a counter hash of seed and t) three cases: a and b with
// random significands and signs, |a| in [2^-61, 2^47] and |b| in
// [2^-100, 2^39] (quotients outside [2^-100, 2^100] are skipped); a quotient
// within two ulps of the midpoint above a random float in [2^-8, 64] (the
// hardest case for rounding); and b a random float with a = b * k for a small
// integer k (quotients at integers, where the rows' round-up conversion
// turns).  Counts the trials whose results differ in any bit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t check_hash(unsigned long long x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return (uint32_t)x;
}

// random float with biased exponent 127 + [lo, hi], random significand and sign
__device__ __forceinline__ float check_float(unsigned long long s, int lo, int hi)
{
    const uint32_t h = check_hash(s), g = check_hash(s * 0x9E3779B97F4A7C15ull + 7u);
    const int e = lo + (int)(g % (uint32_t)(hi - lo + 1));
    return __uint_as_float(((uint32_t)(e + 127) << 23) | (h & 0x807FFFFFu));
}

__global__ void k_check_division(unsigned long long trials, unsigned long long seed,
                                 unsigned long long *mismatches, unsigned long long *checked)
{
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    unsigned long long bad = 0, n = 0;
    for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < trials;
         t += stride) {
        const unsigned long long s = (seed << 40) ^ (t * 4u);
        // 1. random operands
        {
            const float a = check_float(s, -61, 46), b = check_float(s + 1u, -100, 38);
            const float q = __fdiv_rn(a, b);
            const float aq = fabsf(q);
            if (aq >= 0x1p-100f && aq <= 0x1p100f) {
                ++n;
                if (__float_as_uint(div_by_rcp(a, b, rcp_nearest(b))) != __float_as_uint(q)) ++bad;
            }
        }
        // 2. quotients next to a rounding midpoint
        {
            const float m = fabsf(check_float(s + 2u, -8, 5));
            const float b = check_float(s + 3u, -60, 38);
            const double mid = 0.5 * ((double)m + (double)__uint_as_float(__float_as_uint(m) + 1u));
            float a = (float)(mid * (double)b);
            const int k = (int)(check_hash(s + 5u) % 5u) - 2;
            a = __uint_as_float(__float_as_uint(a) + (uint32_t)k);
            const float q = __fdiv_rn(a, b);
            const float aq = fabsf(q);
            if (aq >= 0x1p-100f && aq <= 0x1p100f && fabsf(a) <= 0x1p47f && fabsf(a) >= 0x1p-61f) {
                ++n;
                if (__float_as_uint(div_by_rcp(a, b, rcp_nearest(b))) != __float_as_uint(q)) ++bad;
            }
        }
        // 3. quotients at and next to small integers
        {
            const float b = check_float(s + 6u, -40, 38);
            const int k = (int)(check_hash(s + 7u) % 130u) - 65;
            float a = __fmul_rn(b, (float)k);
            const int d = (int)(check_hash(s + 8u) % 3u) - 1;
            if (a != 0.0f) a = __uint_as_float(__float_as_uint(a) + (uint32_t)d);
            const float q = __fdiv_rn(a, b);
            const float aq = fabsf(q);
            if ((aq >= 0x1p-100f || q == 0.0f) && aq <= 0x1p100f && fabsf(a) <= 0x1p47f &&
                (fabsf(a) >= 0x1p-61f || a == 0.0f)) {
                ++n;
                if (__float_as_uint(div_by_rcp(a, b, rcp_nearest(b))) != __float_as_uint(q)) ++bad;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        bad += __shfl_xor_sync(kFullWarp, bad, o);
        n += __shfl_xor_sync(kFullWarp, n, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (bad) atomicAdd(mismatches, bad);
        atomicAdd(checked, n);
    }
}

__global__ void k_check_reciprocal(unsigned long long *mismatches, unsigned long long *checked)
{
    constexpr unsigned long long kValues = 140ull << 23;   // biased exponents 27 .. 166
    unsigned long long bad = 0, n = 0;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < kValues;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint32_t bits = ((uint32_t)(27u + (i >> 23)) << 23) | (uint32_t)(i & 0x7FFFFFu);
        const float b = __uint_as_float(bits), nb = __uint_as_float(bits | 0x80000000u);
        bad += __float_as_uint(rcp_nearest(b)) != __float_as_uint(__frcp_rn(b));
        bad += __float_as_uint(rcp_nearest(nb)) != __float_as_uint(__frcp_rn(nb));
        n += 2;
    }
    for (int o = 16; o > 0; o >>= 1) {
        bad += __shfl_xor_sync(kFullWarp, bad, o);
        n += __shfl_xor_sync(kFullWarp, n, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (bad) atomicAdd(mismatches, bad);
        atomicAdd(checked, n);
    }
}

cudaError_t check_division(unsigned long long trials, unsigned long long seed, unsigned long long *mismatches,
                           unsigned long long *checked)
{
    unsigned long long *d = nullptr;
    cudaError_t e = cudaMalloc(&d, 2 * sizeof(unsigned long long));
    if (e != cudaSuccess) return e;
    cudaMemset(d, 0, 2 * sizeof(unsigned long long));
    k_check_reciprocal<<<sm_count() * 8, 256>>>(d, d + 1);
    k_check_division<<<sm_count() * 8, 256>>>(trials, seed, d, d + 1);
    e = cudaGetLastError();
    unsigned long long h[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost);
    cudaFree(d);
    *mismatches = h[0];
    *checked = h[1];
    return e;
}

}  // namespace fdzb

// ---------------------------------------------------------------------------
// Allocation-free sort entry point.
//
// Some callers cannot allocate device memory: code running inside a memory
// pool or allocator that forbids cudaMalloc/cudaFree on the hot path, plugins
// whose host process owns every allocation, or real-time loops where an
// allocation (and the device synchronisation cudaFree implies) is not allowed.
// For them, fdzb_sort_pairs_noalloc sorts with a fixed scratch area compiled
// into the library as a file-scope device array: every GPU that loads the
// library holds it (kNoAllocBytes = 8,917,264 bytes: 8.92 MB, 8.50 MiB)
// until the process exits.
//
// The array is a device symbol: in host code its name is only a stand-in, so
// the first call on each device looks up its device address with
// cudaGetSymbolAddress (with that device current) and passes the pointer to the
// kernels.  That first call should therefore come before any stream capture.
// All calls share the array and it keeps the last call's contents, so every
// call starts by clearing, on its stream, the histogram, tickets, error word
// and the look-back words of the tiles it uses; the look-back tags are then
// just the pass numbers, and nothing a call does depends on host-side state
// left by earlier calls.  Calls that overlap on the GPU (two streams, two host
// threads on one device) race on the array.
// ---------------------------------------------------------------------------
namespace fdzb {
namespace {

constexpr int kNoAllocMaxPairs = 1 << 20;   // FDZB_NOALLOC_SORT_MAX_PAIRS
constexpr int kNoAllocTiles = (kNoAllocMaxPairs + kSortTile - 1) / kSortTile;
constexpr size_t kNoAllocKeysOff = 0;
constexpr size_t kNoAllocValsOff = kNoAllocKeysOff + 4ull * kNoAllocMaxPairs;
constexpr size_t kNoAllocHistOff = kNoAllocValsOff + 4ull * kNoAllocMaxPairs;
constexpr size_t kNoAllocTicketOff = kNoAllocHistOff + 4ull * 4 * kRadix;
constexpr size_t kNoAllocErrOff = kNoAllocTicketOff + 4ull * 4;
constexpr size_t kNoAllocStatusOff = kNoAllocErrOff + 256;
constexpr size_t kNoAllocBytes = kNoAllocStatusOff + 8ull * kNoAllocTiles * kRadix;
static_assert(kNoAllocBytes == 8917264, "scratch size quoted in the comments and the header");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char *g_noalloc_ptr[kNoAllocMaxDevices];

__global__ void k_noalloc_status(const int *err, int32_t *status)
{
    *status = *err;
}

// True if the byte ranges [a, a + na) and [b, b + nb) share a byte.
bool overlaps(const void *a, size_t na, const void *b, size_t nb)
{
    const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
    return na && nb && x < y + nb && y < x + na;
}

}  // namespace
}  // namespace fdzb

extern "C" int fdzb_sort_pairs_noalloc(const uint32_t *d_keys_in, const uint32_t *d_vals_in,
                                       uint32_t *d_keys_out, uint32_t *d_vals_out, int32_t n,
                                       uint32_t key_range, void *stream, int32_t *d_status)
{
    using namespace fdzb;
    if (n < 0 || n > kNoAllocMaxPairs)
        return set_error(-1, "fdzb_sort_pairs_noalloc: n must be in [0, 1048576] (the size of its "
                             "built-in scratch area)");
    if (key_range == 0) return set_error(-1, "fdzb_sort_pairs_noalloc: key_range must be positive");
    if (n > 0 && (!d_keys_in || !d_vals_in || !d_keys_out || !d_vals_out))
        return set_error(-1, "fdzb_sort_pairs_noalloc: NULL buffer");
    if (n > 0) {
        // an output may share no byte with an input, the other output or the status word
        const size_t nb = 4ull * (size_t)n;
        const bool bad = overlaps(d_keys_out, nb, d_keys_in, nb) || overlaps(d_keys_out, nb, d_vals_in, nb) ||
                         overlaps(d_keys_out, nb, d_vals_out, nb) || overlaps(d_vals_out, nb, d_keys_in, nb) ||
                         overlaps(d_vals_out, nb, d_vals_in, nb) ||
                         (d_status && (overlaps(d_keys_out, nb, d_status, 4) || overlaps(d_vals_out, nb, d_status, 4)));
        if (bad)
            return set_error(-1, "fdzb_sort_pairs_noalloc: outputs must not overlap the inputs, each other "
                                 "or the status word");
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(-2, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return set_error(-7, "device index out of range");
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess)
                return set_error(-2, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_noalloc_ptr[dev] = (unsigned char *)p;
        }
        base = g_noalloc_ptr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t *tmpK = (uint32_t *)(base + kNoAllocKeysOff);
    uint32_t *tmpV = (uint32_t *)(base + kNoAllocValsOff);
    uint32_t *hist = (uint32_t *)(base + kNoAllocHistOff);
    int *tickets = (int *)(base + kNoAllocTicketOff);
    int *err = (int *)(base + kNoAllocErrOff);
    unsigned long long *status = (unsigned long long *)(base + kNoAllocStatusOff);
    const long long tiles = ((long long)n + kSortTile - 1) / kSortTile;
    // histogram, tickets, error word and the look-back words of the tiles in
    // use start at zero every call (one contiguous range, at most 0.5 MiB)
    e = cudaMemsetAsync(hist, 0, kNoAllocStatusOff - kNoAllocHistOff + 8ull * kRadix * (size_t)tiles, s);
    if (e != cudaSuccess) return set_error(-2, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    const int passes = sort_passes_for((long long)key_range);
    if (n > 0) {
        const int sm = sm_count();
        k_radix_hist<<<grid_for(n, kSortThreads, sm * 4), kSortThreads, 0, s>>>(d_keys_in, nullptr, n, n,
                                                                                  passes, 0, hist);
        // destinations alternate so that the last pass lands in the outputs
        const int grid = grid_for(tiles * kSortThreads, kSortThreads, sm * 4);
        const uint32_t *ki = d_keys_in, *vi = d_vals_in;
        for (int p = 0; p < passes; ++p) {
            const bool toOut = ((passes - 1 - p) % 2) == 0;
            uint32_t *ko = toOut ? d_keys_out : tmpK;
            uint32_t *vo = toOut ? d_vals_out : tmpV;
            // tag p + 1: the cleared words (tag 0) and the words of this call's
            // earlier passes both read as unpublished
            k_radix_pass<true><<<grid, kSortThreads, 0, s>>>(ki, vi, ko, vo, nullptr, n, n, 8 * p,
                                                       hist + p * kRadix, status, nullptr, (uint32_t)p + 1u,
                                                       tickets + p, err);
            ki = ko;
            vi = vo;
        }
    }
    if (d_status) k_noalloc_status<<<1, 1, 0, s>>>(err, d_status);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(-2, std::string("kernel launch: ") + cudaGetErrorString(e));
    return 0;
}
