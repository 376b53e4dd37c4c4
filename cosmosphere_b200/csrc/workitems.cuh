/*
 * workitems.cuh -- the dynamic work queue of the pair kernels.
 *
 * A pass over the leaves is cut into work items, one per group of up to 32 active
 * particles of a leaf's 64-slot window; leaves whose j-stream is long are cut into smaller
 * groups so that no single warp carries a pass's tail.  A persistent grid of warps takes
 * items from a global counter.
 */
#pragma once

#include "pairstream.cuh"
#include "state.hpp"

namespace cosmo {

namespace {

// Zero the per-iteration counters of the Newton work queue and the leaf re-queue flags.
__global__ void begin_iteration_kernel(DevScalars* __restrict__ ds, int* __restrict__ leafNext, int nL,
                                       const int* __restrict__ nLp = nullptr)
{
    if (nLp) nL = *nLp;   // the leaf count on the device (a captured graph)
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0)
    {
        ds->nextActive = 0;
        ds->unconverged = 0;
        ds->listStale = 0;
        ds->workCounter[0] = 0;
        ds->itemsHeavy = 0;
        ds->itemsLight = 0;
        ds->rowParticles = 0;
        ds->settling = 0;
    }
    for (int l = t; l < nL; l += gridDim.x * blockDim.x) leafNext[l] = 0;
}

// Work items of one pass.  The active particles (unconverged ones in a Newton iteration;
// all when converged is null, of all leaves when leaves is null) of each 64-slot window of
// a leaf are grouped, and each group of up to 32 is one item: (leaf, window << 16 | 1, the
// two halves of the group's member mask).  A leaf whose gather list streams more than
// kSplitStream particles is cut into smaller groups, about kSplitWork / stream particles
// each, so that no single warp carries the pass's tail; cut items are queued from the
// front of the buffer and run first (their warps scan the tree for their own box), whole
// groups from the back.  A window's items hold at most its active particles, so cap = the
// particle count always suffices.  The batched form sets both figures per set (tuned).
constexpr uint32_t kSplitStream = 4096;
constexpr uint32_t kSplitWork = 32u * 4096u;
constexpr double kGroupSpread = 1.5;
constexpr uint32_t kStreamUnbounded = 0xffffffffu;   // jstream of a leaf whose walk stopped at the cap
constexpr int kSpreadGroups = 1;   // at least this many h-ordered groups in a spread window

// The cut of one leaf: x = the stream above which it is cut, y = the work of one cut group
// (the same for every leaf; kSplitStream and kSplitWork unless the caller sets others).
struct FixedSplit
{
    uint32_t stream = kSplitStream, work = kSplitWork;
    __device__ __forceinline__ uint2 operator()(int) const { return make_uint2(stream, work); }
};

// The cut of a forest leaf: its set's entry of a per-set table.
struct SetSplit
{
    const int* __restrict__ leafSet;
    const uint2* __restrict__ setSplit;
    __device__ __forceinline__ uint2 operator()(int leaf) const { return setSplit[leafSet[leaf]]; }
};

// Row classification (optional): with rowCount given, an active particle whose
// neighbour row is complete for its current h (count <= K and h <= rowH) goes to
// rowItems (ds->rowParticles of them) instead of a group.
struct RowSplit
{
    const int* __restrict__ rowCount;
    const double* __restrict__ rowH;
    int K;
    int* __restrict__ rowItems;
};

template<class Ranges, class Split = FixedSplit>
__device__ __forceinline__ void plan_items(const int* __restrict__ leaves, int nActive, Ranges ranges,
                                           const int* __restrict__ converged, const uint32_t* __restrict__ jstream,
                                           const double4* __restrict__ xyzh, int4* __restrict__ items, int cap,
                                           DevScalars* __restrict__ ds, RowSplit rs = RowSplit{nullptr, nullptr, 0,
                                                                                              nullptr},
                                           Split split = Split{}, int spreadGroups = kSpreadGroups)
{
    // The block's warps take one leaf each per step and reserve their rows and items
    // together: each warp's counts go to shared memory, one thread makes one global
    // reservation per counter for the block, and each warp writes at its share of it
    // (one atomic per block and counter instead of one per warp and window: the counters
    // are single addresses that every warp of the grid adds to).
    __shared__ int sCnt[3][32];   // per warp: row particles, cut groups, whole groups
    __shared__ int sBase[3];
    __shared__ int sWin[32];
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const int wib = threadIdx.x >> 5, nWib = blockDim.x >> 5;
    for (int w0 = blockIdx.x * nWib; w0 < nActive; w0 += gridDim.x * nWib)
    {
        const int w = w0 + wib;
        const bool have = w < nActive;
        const int leaf = have ? (leaves ? leaves[w] : w) : 0;
        const uint2 rg = have ? ranges(leaf) : make_uint2(0u, 0u);
        const uint32_t p0 = rg.x, p1 = rg.y;
        const uint32_t S = have ? jstream[leaf] : 0u;
        const uint2 cut = split(leaf);
        const int gsize = S <= cut.x ? 32 : max(1, int(cut.y / S));
        if (lane == 0) sWin[wib] = int((p1 - p0 + 63) >> 6);
        __syncthreads();
        int rounds = 0;
        for (int k = 0; k < nWib; ++k) rounds = max(rounds, sWin[k]);
        __syncthreads();   // sWin is written again by the next step
        for (int r = 0; r < rounds; ++r)
        {
            const uint32_t g = p0 + 64u * uint32_t(r);
            const bool win = g < p1;   // warp-uniform
            const uint32_t a0 = g + lane, a1 = g + 32 + lane;
            bool act0 = win && a0 < p1 && (!converged || converged[a0] == 0);
            bool act1 = win && a1 < p1 && (!converged || converged[a1] == 0);
            bool row0 = false, row1 = false;
            if (rs.rowCount != nullptr)
            {
                auto rowOK = [&](uint32_t a) {
                    return unsigned(rs.rowCount[a]) <= unsigned(rs.K) && xyzh[a].w <= rs.rowH[a];
                };
                row0 = act0 && rowOK(a0);
                row1 = act1 && rowOK(a1);
                act0 = act0 && !row0;
                act1 = act1 && !row1;
            }
            const uint32_t q0 = __ballot_sync(0xffffffffu, row0), q1 = __ballot_sync(0xffffffffu, row1);
            const uint32_t c0 = __ballot_sync(0xffffffffu, act0), c1 = __ballot_sync(0xffffffffu, act1);
            const int nC = __popc(c0) + __popc(c1);
            const int wnd = win ? int((g - p0) >> 6) : 0;
            const int whole = (nC + 31) >> 5;
            // A window whose smoothing lengths spread by more than kGroupSpread is grouped by
            // h (ranks in ascending h), into at least spreadGroups groups and however many
            // its count and cut need: a group's box is set by its widest particle, so the
            // narrow ones keep a box nearer their own size (measured on B200 for the Plummer
            // workload: at least one group, i.e. h order only where a window needs two or
            // more anyway, is fastest; forcing 2, 4 or 8 costs more in groups than it saves
            // in tests).  Grouping changes no result (every particle's sums run over the same
            // pairs in j order).
            const double inf = __longlong_as_double(0x7ff0000000000000ll);
            const double h0 = act0 ? xyzh[a0].w : inf, h1 = act1 ? xyzh[a1].w : inf;
            const double hmin = warp_min(fmin(h0, h1));
            const double hmax = warp_max(fmax(act0 ? h0 : 0.0, act1 ? h1 : 0.0));
            const bool byH = nC > 1 && hmax > kGroupSpread * hmin;
            const int cutG = (nC + gsize - 1) / gsize;
            const int G = nC == 0 ? 0 : max(byH ? max(whole, min(spreadGroups, nC)) : whole, cutG);
            // cut items (long streams) scan the tree for their box; so do all items of a leaf
            // whose list walk stopped at the stream cap (its list is empty)
            const bool splitW = cutG > whole || S == kStreamUnbounded;
            if (lane == 0)
            {
                sCnt[0][wib] = __popc(q0) + __popc(q1);
                sCnt[1][wib] = splitW ? G : 0;
                sCnt[2][wib] = splitW ? 0 : G;
            }
            __syncthreads();
            if (threadIdx.x < 3)
            {
                // the block's reservation: exclusive prefixes over its warps, one atomic
                const int c = threadIdx.x;
                int run = 0;
                for (int k = 0; k < nWib; ++k)
                {
                    const int v = sCnt[c][k];
                    sCnt[c][k] = run;
                    run += v;
                }
                int* ctr = c == 0 ? &ds->rowParticles : (c == 1 ? &ds->itemsHeavy : &ds->itemsLight);
                sBase[c] = run > 0 ? atomicAdd(ctr, run) : 0;
            }
            __syncthreads();
            if (q0 | q1)
            {
                const int base = sBase[0] + sCnt[0][wib];
                if (row0) rs.rowItems[base + __popc(q0 & lt)] = int(a0);
                if (row1) rs.rowItems[base + __popc(q0) + __popc(q1 & lt)] = int(a1);
            }
            if (G > 0)
            {
                const int base = splitW ? sBase[1] + sCnt[1][wib] : sBase[2] + sCnt[2][wib];
                // group k takes the active ranks [k nC / G, (k + 1) nC / G): in slot order,
                // or in (h, slot) order for a spread window
                int r0 = __popc(c0 & lt), r1 = __popc(c0) + __popc(c1 & lt);
                if (byH)
                {
                    int k0 = 0, k1 = 0;
                    for (int t = 0; t < 32; ++t)
                    {
                        const double u0 = __shfl_sync(0xffffffffu, h0, t), u1 = __shfl_sync(0xffffffffu, h1, t);
                        // slots t and 32 + t against this lane's two slots (inactive slots hold inf)
                        k0 += (u0 < h0 || (u0 == h0 && t < lane)) + (u1 < h0);
                        k1 += (u0 < h1 || u0 == h1) + (u1 < h1 || (u1 == h1 && t < lane));
                    }
                    r0 = k0;
                    r1 = k1;
                }
                for (int k = 0; k < G; ++k)
                {
                    const int lo = k * nC / G, hi = (k + 1) * nC / G;
                    const uint32_t i0 = __ballot_sync(0xffffffffu, act0 && r0 >= lo && r0 < hi);
                    const uint32_t i1 = __ballot_sync(0xffffffffu, act1 && r1 >= lo && r1 < hi);
                    const int idx = splitW ? base + k : cap - 1 - (base + k);
                    if (lane == 0 && idx >= 0 && idx < cap)
                        items[idx] = make_int4(leaf, (wnd << 16) | 1, int(i0), int(i1));
                }
            }
            __syncthreads();   // the shared counts are reused by the next round
        }
    }
}

__global__ void plan_items_kernel(const int* __restrict__ leaves, int nActive, const uint32_t* __restrict__ layout,
                                  const int* __restrict__ converged, const uint32_t* __restrict__ jstream,
                                  const double4* __restrict__ xyzh, int4* __restrict__ items, int cap,
                                  DevScalars* __restrict__ ds,
                                  RowSplit rs = RowSplit{nullptr, nullptr, 0, nullptr},
                                  FixedSplit split = FixedSplit{}, int spreadGroups = kSpreadGroups)
{
    plan_items(leaves, nActive, LayoutRanges{layout}, converged, jstream, xyzh, items, cap, ds, rs, split,
               spreadGroups);
}

// The same with the active-leaf count read on the device (a graph-run Newton loop), and
// the row classification used only once *rowsReady is set.
__global__ void plan_items_count_kernel(const int* __restrict__ leaves, const int* __restrict__ countPtr,
                                        const int* __restrict__ rowsReady, const uint32_t* __restrict__ layout,
                                        const int* __restrict__ converged, const uint32_t* __restrict__ jstream,
                                        const double4* __restrict__ xyzh, int4* __restrict__ items, int cap,
                                        DevScalars* __restrict__ ds, RowSplit rs, FixedSplit split, int spreadGroups)
{
    const RowSplit r = (rowsReady != nullptr && *rowsReady) ? rs : RowSplit{nullptr, nullptr, 0, nullptr};
    plan_items(leaves, *countPtr, LayoutRanges{layout}, converged, jstream, xyzh, items, cap, ds, r, split,
               spreadGroups);
}

// The same over a forest's range table, the active count read on the device, each leaf
// cut by its set's entry of setSplit.
__global__ void plan_items_table_kernel(const int* __restrict__ leaves, const int* __restrict__ countPtr,
                                        const uint2* __restrict__ range, const int* __restrict__ converged,
                                        const uint32_t* __restrict__ jstream, const double4* __restrict__ xyzh,
                                        int4* __restrict__ items, int cap, DevScalars* __restrict__ ds,
                                        const int* __restrict__ leafSet, const uint2* __restrict__ setSplit)
{
    plan_items(leaves, *countPtr, TableRanges{range}, converged, jstream, xyzh, items, cap, ds,
               RowSplit{nullptr, nullptr, 0, nullptr}, SetSplit{leafSet, setSplit});
}

// A persistent grid: as many blocks of the kernel as fit on the device at once.
template<class K>
int persistent_grid(const State& s, K kernel, int threads)
{
    int perSM = 0;
    COSMO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, threads, 0));
    return std::max(1, perSM) * s.numSMs;
}

// Decode of a work item: the group's particles are the active ranks
// [grp * nAct / G, (grp + 1) * nAct / G) of the window starting at g0.
struct Item
{
    int leaf, grp, G, nAct, ng;
    uint32_t g0, m0, m1;
};

__device__ __forceinline__ Item decode_item(const int4& it, uint32_t leafBegin)
{
    Item d;
    d.leaf = it.x;
    const int wnd = it.y >> 16;
    d.grp = (it.y >> 8) & 255;
    d.G = it.y & 255;
    d.m0 = uint32_t(it.z);
    d.m1 = uint32_t(it.w);
    d.nAct = __popc(d.m0) + __popc(d.m1);
    d.ng = (d.grp + 1) * d.nAct / d.G - d.grp * d.nAct / d.G;
    d.g0 = leafBegin + 64u * uint32_t(wnd);
    return d;
}

__device__ __forceinline__ Item decode_item(const int4& it, const uint32_t* __restrict__ layout)
{
    return decode_item(it, layout[it.x]);
}

// Next item index of this warp (lane 0 takes it), or -1 when the queue is empty.  Cut
// items sit at the front of the buffer, whole ones at the back.
__device__ __forceinline__ int next_item(DevScalars* ds, int nHeavy, int nItems, int cap)
{
    int w = 0;
    if ((threadIdx.x & 31) == 0) w = atomicAdd(&ds->workCounter[0], 1);
    w = __shfl_sync(0xffffffffu, w, 0);
    if (w >= nItems) return -1;
    return w < nHeavy ? w : cap - 1 - (w - nHeavy);
}

} // namespace
} // namespace cosmo
