// fdzb_sort.cuh -- stable LSD radix sort of (uint32 key, uint32 value) pairs.
//
// Replaces the reference's thrust::sort_by_key calls
// (K/Step3_bindSampleToBin.inl:125-127, K/Step4_RasterizeTriangleToBin.inl:221-223):
// same result (keys ascending, equal keys in input order), one-sweep design:
//   1. one histogram pass counts the 8-bit digits of every pass at once
//      (shared-memory digit histograms, one global atomic per digit per block);
//   2. one scatter pass per digit: each CTA takes the next tile ticket, ranks its
//      keys with warp match/popc against per-warp shared histograms, publishes its
//      per-digit tile count, and finds its global offsets by a decoupled look-back
//      over the previous tiles' published counts (bounded waits); the tile is
//      reordered by digit in shared memory, then written out in digit runs, so
//      that consecutive threads store to consecutive addresses.
// The element count may live in device memory (n_dev), so the sort is enqueued
// without a host round trip.
#pragma once
#include "fdzb_device.cuh"

namespace fdzb {

#ifndef FDZB_SORT_MINBLOCKS
#define FDZB_SORT_MINBLOCKS 3
#endif
constexpr int kSortThreads = 256;                      // = kRadix: thread d handles digit d
constexpr int kSortItems = FDZB_SORT_ITEMS;
constexpr int kSortTile = kSortThreads * kSortItems;   // keys per tile
constexpr int kRadix = 256;
// Look-back status word: [63:32] launch epoch, [31:30] flag, [29:0] count.  A
// word whose epoch is not the current one reads as "not yet published", so the
// status array never needs clearing between launches or passes.
constexpr unsigned long long kStatAgg = 1ull << 30;
constexpr unsigned long long kStatPrefix = 2ull << 30;
constexpr unsigned long long kStatMask = (1ull << 30) - 1ull;

__device__ __forceinline__ int sort_count(const int *n_dev, int n_static, int cap)
{
    int n = n_dev ? *(volatile const int *)n_dev : n_static;
    return n < cap ? n : cap;
}

// hist[p * 256 + digit] += count, for passes p < passes; pass p's digit is
// bits [shift0 + 8p, shift0 + 8p + 8) of the key.
__global__ void __launch_bounds__(kSortThreads)
    k_radix_hist(const uint32_t *__restrict__ keys, const int *n_dev, int n_static, int cap,
                 int passes, int shift0, uint32_t *__restrict__ hist)
{
    __shared__ uint32_t s_hist[4 * kRadix];
    const int n = sort_count(n_dev, n_static, cap);
    for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t k = keys[i];
        for (int p = 0; p < passes; ++p) atomicAdd(&s_hist[p * kRadix + ((k >> (shift0 + 8 * p)) & 255u)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x)
        if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
}

// One digit pass.  status: [tiles * 256] zeroed before the pass; ticket zeroed.
// KV = false sorts keys alone (vin and vout unused): the pairs' keys can carry
// their value in the bits below the digits.
// SEG = true (the last pass of a sort whose keys name segments, key >> segShift):
// the pass also writes the segment bounds of the sorted output, the restated
// K/binRaster.inl:5-33 -- segStart[k] = first index of segment k, segEnd[k] =
// last index + 1.  A tile holds its elements in final order, so an element that
// begins (ends) a run of its segment inside the tile lowers segStart (raises
// segEnd) of that segment by an atomic; the smallest first and the largest last
// over the tiles are the segment's bounds.  The arrays start at (INT_MAX, 0);
// absent segments keep those and are set to (0, 0) afterwards (k_items).
template <bool KV, int ITEMS = kSortItems, int MINB = FDZB_SORT_MINBLOCKS, bool SEG = false>
__global__ void __launch_bounds__(kSortThreads, MINB)
    k_radix_pass(const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin,
                 uint32_t *__restrict__ kout, uint32_t *__restrict__ vout, const int *n_dev,
                 int n_static, int cap, int shift, const uint32_t *__restrict__ hist,
                 unsigned long long *status, const uint32_t *epochWord, uint32_t epochLo, int *ticket,
                 int *err, int32_t *segStart = nullptr, int32_t *segEnd = nullptr, int segShift = 0,
                 uint32_t nslots = 0)
{
    constexpr int WARPS = kSortThreads / 32;
    constexpr int TILE = kSortThreads * ITEMS;
    __shared__ uint32_t s_start[kRadix];
    __shared__ uint32_t s_whist[WARPS][kRadix];
    __shared__ uint32_t s_base[kRadix];
    __shared__ uint32_t s_tstart[kRadix];
    __shared__ uint32_t s_scan[WARPS];
    __shared__ uint32_t s_k[TILE];
    __shared__ uint32_t s_v[KV ? TILE : 1];
    __shared__ int s_tile;

    const int n = sort_count(n_dev, n_static, cap);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // look-back tag of this pass: 16 x (launch number, a device word that k_init
    // advances, so graph replays get fresh tags) + 4 x sort slot + pass
    const uint32_t epoch = (epochWord ? *epochWord * 16u : 0u) + epochLo;

    // Exclusive scan of this pass's digit histogram (digit = tid).
    {
        uint32_t h = hist[tid];
        uint32_t x = h;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(kFullWarp, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_scan[warp] = x;
        __syncthreads();
        uint32_t wbase = 0;
        for (int w = 0; w < warp; ++w) wbase += s_scan[w];
        s_start[tid] = wbase + x - h;
    }

    for (;;) {
        __syncthreads();
        if (tid == 0) s_tile = atomicAdd(ticket, 1);
        for (int i = tid; i < WARPS * kRadix; i += kSortThreads) (&s_whist[0][0])[i] = 0;
        __syncthreads();
        const int tile = s_tile;
        if ((long long)tile * TILE >= n) break;
        const int tileN = min(TILE, n - tile * TILE);

        const int base = tile * TILE + warp * (ITEMS * 32);
        uint32_t k[ITEMS], v[ITEMS], rk[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const int idx = base + i * 32 + lane;
            const bool ok = idx < n;
            k[i] = ok ? kin[idx] : 0u;
            v[i] = (KV && ok) ? vin[idx] : 0u;
        }
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const int idx = base + i * 32 + lane;
            const bool ok = idx < n;
            const uint32_t d = ok ? ((k[i] >> shift) & 255u) : 256u;
            const uint32_t peers = __match_any_sync(kFullWarp, d);
            const uint32_t lt = peers & lanemask_lt();
            uint32_t before = ok ? s_whist[warp][d] : 0u;
            __syncwarp();
            if (ok && lt == 0) s_whist[warp][d] = before + __popc(peers);
            __syncwarp();
            rk[i] = before + __popc(lt);
        }
        __syncthreads();

        // Per digit: prefix over warps, tile total, and the digit's start in the tile.
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < WARPS; ++w) {
            uint32_t c = s_whist[w][tid];
            s_whist[w][tid] = run;
            run += c;
        }
        {
            uint32_t x = run;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(kFullWarp, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) s_scan[warp] = x;
            __syncthreads();
            uint32_t wbase = 0;
            for (int w = 0; w < warp; ++w) wbase += s_scan[w];
            s_tstart[tid] = wbase + x - run;
        }
        // Decoupled look-back on digit tid.
        unsigned long long *my = status + (size_t)tile * kRadix + tid;
        const unsigned long long ep = (unsigned long long)epoch << 32;
        uint32_t excl = 0;
        if (tile == 0) {
            st_volatile_u64(my, ep | kStatPrefix | run);
        } else {
            st_volatile_u64(my, ep | kStatAgg | run);
            int t = tile - 1;
            unsigned spins = 0;
            while (t >= 0) {
                const unsigned long long s = ld_volatile_u64(status + (size_t)t * kRadix + tid);
                const unsigned long long flag = ((s >> 32) == epoch) ? (s & 0xC0000000ull) : 0ull;
                if (flag == 0) {
                    if (++spins > kSpinLimit) {
                        atomicOr(err, (int)ERR_LOOKBACK_TIMEOUT);
                        break;
                    }
                    continue;
                }
                excl += (uint32_t)(s & kStatMask);
                if (flag == kStatPrefix) break;
                --t;
            }
            st_volatile_u64(my, ep | kStatPrefix | (excl + run));
        }
        // global position of the tile's first element with digit tid
        s_base[tid] = s_start[tid] + excl;
        __syncthreads();

        // reorder the tile by digit in shared memory (stable)
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const int idx = base + i * 32 + lane;
            if (idx < n) {
                const uint32_t d = (k[i] >> shift) & 255u;
                const uint32_t lp = s_tstart[d] + s_whist[warp][d] + rk[i];
                s_k[lp] = k[i];
                if (KV) s_v[lp] = v[i];
            }
        }
        __syncthreads();
        // write out: element j of the reordered tile goes to s_base[d] + (j - s_tstart[d])
        for (int j = tid; j < tileN; j += kSortThreads) {
            const uint32_t kk = s_k[j];
            const uint32_t d = (kk >> shift) & 255u;
            const uint32_t dst = s_base[d] + ((uint32_t)j - s_tstart[d]);
            if (dst < (uint32_t)cap) {
                kout[dst] = kk;
                if (KV) vout[dst] = s_v[j];
                if (SEG) {
                    const uint32_t sg = kk >> segShift;
                    if (sg >= nslots) {
                        atomicOr(err, (int)ERR_INTERNAL);
                    } else {
                        if (j == 0 || (s_k[j - 1] >> segShift) != sg) atomicMin(&segStart[sg], (int)dst);
                        if (j == tileN - 1 || (s_k[j + 1] >> segShift) != sg) atomicMax(&segEnd[sg], (int)dst + 1);
                    }
                }
            }
        }
    }
}

}  // namespace fdzb
