/*
 * batch.cu -- many independent particle sets solved together: one segmented sort, one
 * forest, and ONE density launch per Newton-Raphson iteration across every set.
 *
 * The sets are concatenated set-major (set s owns [off[s], off[s+1])).  Each set keeps its
 * own box, keys, leaf tree (split while a node holds more than that set's bucket size),
 * pre-order node range and j-leaf lists; a set's leaves and nodes are contiguous in the
 * forest and its walks never leave its node range.  The Newton kernel takes i-leaves
 * from all sets through one work list; each leaf carries its set's mass, periodicity and
 * box.  Per particle, the arithmetic is the single-set form's (plain FP64 or mixed), and
 * the j order is ascending sorted index, so a set solved in a batch gives the same h and
 * rho as the same set solved alone.
 */
#include <algorithm>
#include <cstring>
#include <string>

#include "densengine.cuh"
#include "pairstream.cuh"
#include "sort.cuh"
#include "state.hpp"
#include "workitems.cuh"
#include "../../include/cosmosphere.h"

namespace cosmo {

// Newton-loop state kept on the device, so the loop body needs no host reads.
struct LoopState
{
    int nActiveLeaves, nActiveParticles, iter, maxIter, nAll, pad[3];
    long long activePerIter[128];
};

struct Batch
{
    State core;                       // stream, device scalars, scratch for sort and scan
    int nsets = 0, n = 0, nLeaves = 0, numNodes = 0, itersRun = 0, unconverged = 0;
    std::vector<int> offs;            // host copy, nsets + 1
    std::vector<long long> activePerIter;
    double tBuild = 0, tNR = 0, tList = 0, tTotal = 0;
    unsigned long long pairs = 0;
    DBuf<int> dOffs, setOf, nAliveSet, setLeafStart, setNodeStart, bucket, setPer;
    DBuf<double> setMargin;           // per set: gather-radius widening of its lists
    DBuf<uint2> setSplit;             // per set: stream above which a leaf is cut, work per cut group
    DBuf<double> ux, uy, uz, uh, pmass, setBox6, rho, gradh, hmaxLeaf;
    DBuf<double4> xyzh, preCenter, preHalf;
    DBuf<int> converged, orderA, orderB, leafSet, leafSet2, leafPre, preLeaf, preSkip, jlist, activeA, activeB, allLeaves;
    DBuf<uint64_t> keysA, keysB, leafKey, leafKey2;
    DBuf<uint32_t> ops, opsScan, nodeCount, leafPreStart, jcount, jOffset, setHist, setBase, jstream;
    DBuf<uint32_t> jcountPrev, jOffsetPrev;   // the previous walk's lists, kept for reuse
    DBuf<int> jlistPrev, walked, walkScratch;
    DBuf<double> listH;                       // h each leaf's list covers (0: none)
    DBuf<int4> items;                 // Newton work items (leaf, window|group|G, m0, m1)
    DBuf<int> leafNext;               // leaf already queued for the next iteration
    DBuf<uint2> leafRange;
    DBuf<DevBox> boxes;
    DBuf<LoopState> loop;
    uint32_t listCap = 0;
    std::vector<double> tuning;       // per set: bucket, list margin, cut stream, cut work
    bool graphUsed = false;
};

namespace {

Batch& batch()
{
    static Batch* b = new Batch();   // deliberately leaked, as the single-set state
    return *b;
}

constexpr int kWarpsPerBlock = 4;
constexpr int kThreads = 32 * kWarpsPerBlock;
constexpr double kBatchListMargin = 1.15;   // default gather-radius widening of a set's lists
constexpr int kMinTuneBucket = 8, kMaxTuneBucket = 1024;   // leaf capacities a set may be given
constexpr int kWalkScratchB = 128;   // list entries per leaf the count pass keeps for the fill

__device__ __forceinline__ int set_of_pos(const int* __restrict__ offs, int nsets, long k)
{
    int lo = 0, hi = nsets;   // last s with offs[s] <= k
    while (hi - lo > 1)
    {
        const int mid = (lo + hi) >> 1;
        if (offs[mid] <= k) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void setof_kernel(const int* __restrict__ offs, int nsets, int n, int* __restrict__ setOf)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) setOf[i] = set_of_pos(offs, nsets, i);
}

// One block per set: the periodic box as given, or the open-boundary padded cube of the
// single-set build (src/tree.cu:54-72) over this set's particles.
__global__ void set_box_kernel_b(const int* __restrict__ offs, const int* __restrict__ per,
                                 const double* __restrict__ box6, const double* __restrict__ x,
                                 const double* __restrict__ y, const double* __restrict__ z, DevBox* __restrict__ boxes)
{
    const int s = blockIdx.x;
    const int a = offs[s], b = offs[s + 1];
    __shared__ double sm[32][6];
    if (per[s])
    {
        if (threadIdx.x == 0)
        {
            DevBox bx;
            for (int d = 0; d < 3; ++d) { bx.lo[d] = box6[6 * s + 2 * d]; bx.hi[d] = box6[6 * s + 2 * d + 1]; }
            bx.periodic = 1;
            box_finish(bx);
            boxes[s] = bx;
        }
        return;
    }
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = a + threadIdx.x; i < b; i += blockDim.x)
    {
        const double c[3] = {x[i], y[i], z[i]};
        for (int d = 0; d < 3; ++d) { mn[d] = fmin(mn[d], c[d]); mx[d] = fmax(mx[d], c[d]); }
    }
    for (int o = 16; o > 0; o >>= 1)
        for (int d = 0; d < 3; ++d)
        {
            mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
            mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int d = 0; d < 3; ++d) { sm[w][d] = mn[d]; sm[w][3 + d] = mx[d]; }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        for (int d = 0; d < 3; ++d) { mn[d] = sm[0][d]; mx[d] = sm[0][3 + d]; }
        for (int ww = 1; ww < int(blockDim.x >> 5); ++ww)
            for (int d = 0; d < 3; ++d) { mn[d] = fmin(mn[d], sm[ww][d]); mx[d] = fmax(mx[d], sm[ww][3 + d]); }
        const double sx = mx[0] - mn[0], sy = mx[1] - mn[1], sz = mx[2] - mn[2];
        double span = (sx < sy) ? sy : sx;
        span = (span < sz) ? sz : span;
        span = span * 1.00001;
        const double half = 0.5 * span;
        DevBox bx;
        for (int d = 0; d < 3; ++d)
        {
            const double ctr = 0.5 * (mn[d] + mx[d]);
            bx.lo[d] = ctr - half;
            bx.hi[d] = ctr + half;
        }
        bx.periodic = 0;
        box_finish(bx);
        boxes[s] = bx;
    }
}

__global__ void keys_kernel_b(const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, const double* __restrict__ h, const int* __restrict__ setOf,
                              int n, const DevBox* __restrict__ boxes, uint64_t* __restrict__ keys)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DevBox b = boxes[setOf[i]];
    uint64_t k = kDeadKey;
    if (h[i] > 0.0)
        k = hilbert_key(quantise(x[i], b.lo[0], b.scale[0]), quantise(y[i], b.lo[1], b.scale[1]),
                        quantise(z[i], b.lo[2], b.scale[2]));
    keys[i] = k;
}

__global__ void set_hist_kernel(const int* __restrict__ setOf, int n, int shift, uint32_t* __restrict__ hist)
{
    __shared__ uint32_t s[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) s[i] = 0;
    __syncthreads();
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        atomicAdd(&s[(uint32_t(setOf[i]) >> shift) & 255u], 1u);
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (s[i]) atomicAdd(&hist[i], s[i]);
}

// nAlive of every set: the first dead key of the set's (sorted) segment.
__global__ void alive_kernel_b(const uint64_t* __restrict__ keys, const int* __restrict__ offs, int nsets, int n,
                               int* __restrict__ nAlive)
{
    const long k = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int s = set_of_pos(offs, nsets, k);
    const long a = offs[s], b = offs[s + 1];
    const bool dead = keys[k] == kDeadKey;
    const bool prevAlive = (k == a) ? true : keys[k - 1] != kDeadKey;
    if (dead && prevAlive) nAlive[s] = int(k - a);
    if (!dead && k == b - 1) nAlive[s] = int(b - a);
}

__global__ void gather_kernel_b(const int* __restrict__ order, int n, const double* __restrict__ ux,
                                const double* __restrict__ uy, const double* __restrict__ uz,
                                const double* __restrict__ uh, double4* __restrict__ xyzh)
{
    const long k = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = order[k];
    xyzh[k] = make_double4(ux[i], uy[i], uz[i], uh[i]);
}

__device__ __forceinline__ uint32_t lower_bound_u64b(const uint64_t* a, uint32_t n, uint64_t v)
{
    uint32_t lo = 0, hi = n;
    while (lo < hi)
    {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint64_t leaf_end(const uint64_t* key, const int* set, int L, int l)
{
    return (l + 1 < L && set[l + 1] == set[l]) ? key[l + 1] : kKeyEnd;
}

__global__ void roots_kernel(int nsets, uint64_t* __restrict__ key, int* __restrict__ set)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nsets) { key[s] = 0; set[s] = s; }
}

__global__ void leaf_count_kernel_b(const uint64_t* __restrict__ key, const int* __restrict__ set, int L,
                                    const uint64_t* __restrict__ keys, const int* __restrict__ offs,
                                    const int* __restrict__ nAlive, const int* __restrict__ bucket,
                                    uint32_t* __restrict__ ops, uint2* __restrict__ range)
{
    const long l = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (l >= L) return;
    const int s = set[l];
    const uint64_t a = key[l], b = leaf_end(key, set, L, int(l));
    const uint32_t base = uint32_t(offs[s]), na = uint32_t(nAlive[s]);
    const uint32_t lo = lower_bound_u64b(keys + base, na, a), hi = lower_bound_u64b(keys + base, na, b);
    range[l] = make_uint2(base + lo, base + hi);
    const int lev = level_of_range(b - a);
    ops[l] = (hi - lo > uint32_t(bucket[s]) && lev < kMaxLevel) ? 8u : 1u;
}

__global__ void leaf_split_kernel_b(const uint64_t* __restrict__ key, const int* __restrict__ set, int L,
                                    const uint32_t* __restrict__ ops, const uint32_t* __restrict__ pos,
                                    uint64_t* __restrict__ key2, int* __restrict__ set2)
{
    const long l = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (l >= L) return;
    const uint64_t a = key[l];
    const uint32_t p = pos[l];
    const int s = set[l];
    if (ops[l] == 8u)
    {
        const uint64_t child = (leaf_end(key, set, L, int(l)) - a) >> 3;
        for (int o = 0; o < 8; ++o) { key2[p + o] = a + uint64_t(o) * child; set2[p + o] = s; }
    }
    else { key2[p] = a; set2[p] = s; }
}

__global__ void set_leaf_start_kernel(const int* __restrict__ set, int L, int nsets, int* __restrict__ start)
{
    const long l = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (l > L) return;
    if (l == L) { start[nsets] = L; return; }
    if (l == 0 || set[l - 1] != set[l]) start[set[l]] = int(l);
}

__device__ __forceinline__ int first_aligned_level_b(uint64_t k)
{
    if (k == 0) return 0;
    const int L0 = kMaxLevel - (__ffsll((long long)k) - 1) / 3;
    return L0 < 0 ? 0 : L0;
}

__global__ void node_count_kernel_b(const uint64_t* __restrict__ key, const int* __restrict__ set, int L,
                                    uint32_t* __restrict__ cnt)
{
    const long l = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (l >= L) return;
    const uint64_t k = key[l];
    const int lev = level_of_range(leaf_end(key, set, L, int(l)) - k);
    const int L0 = first_aligned_level_b(k);
    cnt[l] = uint32_t((lev > L0 ? lev - L0 : 0) + 1);
}

__global__ void set_node_start_kernel(const int* __restrict__ setLeafStart, const uint32_t* __restrict__ leafPreStart,
                                      int nsets, int* __restrict__ setNodeStart)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s <= nsets) setNodeStart[s] = int(leafPreStart[setLeafStart[s]]);
}

// Pre-order emission per leaf, as the single-set build, with subtree ends and geometry
// taken within the leaf's own set.
__global__ void node_emit_kernel_b(const uint64_t* __restrict__ key, const int* __restrict__ set, int L,
                                   const uint32_t* __restrict__ start, const int* __restrict__ setLeafStart,
                                   const int* __restrict__ setNodeStart, const DevBox* __restrict__ boxes,
                                   int* __restrict__ preLeaf, int* __restrict__ preSkip, int* __restrict__ leafPre,
                                   double4* __restrict__ preCenter, double4* __restrict__ preHalf)
{
    const long l = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (l >= L) return;
    const int s = set[l];
    const uint64_t k = key[l];
    const int lev = level_of_range(leaf_end(key, set, L, int(l)) - k);
    const int L0 = first_aligned_level_b(k);
    const int ls = setLeafStart[s], le = setLeafStart[s + 1];
    const DevBox bx = boxes[s];
    uint32_t pos = start[l];
    for (int a = (L0 < lev ? L0 : lev); a <= lev; ++a, ++pos)
    {
        preLeaf[pos] = (a == lev) ? int(l) : -1;
        const uint64_t end = k + node_range(a);
        // first leaf of this set starting at or after end
        int lo = ls, hi = le;
        while (lo < hi)
        {
            const int mid = (lo + hi) >> 1;
            if (key[mid] < end) lo = mid + 1;
            else hi = mid;
        }
        const uint32_t next = (end >= kKeyEnd || lo >= le) ? uint32_t(setNodeStart[s + 1]) : start[lo];
        preSkip[pos] = int(next - pos);
        uint32_t ic[3];
        hilbert_cell(k, ic[0], ic[1], ic[2]);
        const uint32_t side = 1u << (kMaxLevel - a);
        const double sd = double(side);
        double c[3], h[3];
        for (int d = 0; d < 3; ++d)
        {
            const double corner = double(ic[d] & ~(side - 1u));
            c[d] = bx.lo[d] + (corner + 0.5 * sd) * bx.unit[d];
            h[d] = 0.5 * sd * bx.unit[d];
        }
        preCenter[pos] = make_double4(c[0], c[1], c[2], 0.0);
        preHalf[pos] = make_double4(h[0], h[1], h[2], 0.0);
        if (a == lev) leafPre[l] = int(pos);
    }
}

__global__ void hmax_leaf_kernel_b(const double4* __restrict__ xyzh, const uint2* __restrict__ range,
                                   const int* __restrict__ leaves, const int* __restrict__ countPtr,
                                   double* __restrict__ hmax)
{
    const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= *countPtr) return;
    const int l = leaves[t];
    const uint2 r = range[l];
    double hm = 0.0;
    for (uint32_t j = r.x; j < r.y; ++j)
    {
        const double hj = xyzh[j].w;
        if (isfinite(hj)) hm = fmax(hm, hj);
    }
    hmax[l] = hm;
}

// Gather walk of one i-leaf over its own set's pre-order nodes (the single-set walk's
// window scan, include/tree.cuh:228-389 accept test).
template<bool Fill>
__global__ void __launch_bounds__(256)
list_walk_kernel_b(const int* __restrict__ leaves, const int* __restrict__ countPtr, const int* __restrict__ set,
                   const int* __restrict__ setNodeStart,
                   const int* __restrict__ leafPre, const double* __restrict__ hmaxLeaf,
                   const double4* __restrict__ preCenter, const double4* __restrict__ preHalf,
                   const int* __restrict__ preSkip, const int* __restrict__ preLeaf, const DevBox* __restrict__ boxes,
                   uint32_t* __restrict__ jcount, const uint32_t* __restrict__ jOffset, int* __restrict__ jlist,
                   uint32_t listCap, int* err, const uint2* __restrict__ range, uint32_t* __restrict__ jstream,
                   double* __restrict__ listH, int* __restrict__ walked, const uint32_t* __restrict__ jcountPrev,
                   const uint32_t* __restrict__ jOffsetPrev, const int* __restrict__ jlistPrev,
                   const double* __restrict__ setMargin, int* __restrict__ scratch)
{
    const int lane = threadIdx.x & 31;
    const int nAct = *countPtr;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nAct; t += (gridDim.x * blockDim.x) >> 5)
    {
    const int leaf = leaves[t];
    double hm = hmaxLeaf[leaf];
    if (!isfinite(hm) || hm <= 0.0) hm = 0.0;
    // A list built at the set's margin x an earlier hmax and kept by the previous walk is
    // a superset, in the same ascending order, of the list this hmax needs: it is copied
    // instead of walked.
    if (!Fill)
    {
        const bool reuse = hm <= listH[leaf] && jcountPrev[leaf] > 0;
        if (reuse)
        {
            if (lane == 0) { jcount[leaf] = jcountPrev[leaf]; walked[leaf] = 0; }
            continue;
        }
    }
    else if (walked[leaf] != 0)
    {
        // a walked list that fitted in the count pass's copy is copied, not walked again
        const uint32_t dst = jOffset[leaf], cnt = jOffset[leaf + 1] - dst;
        if (cnt <= uint32_t(kWalkScratchB))
        {
            if (jOffset[leaf + 1] > listCap)
            {
                if (lane == 0) atomicOr(err, int(kErrListFull));
                continue;
            }
            const int* src = scratch + size_t(leaf) * kWalkScratchB;
            for (uint32_t k = lane; k < cnt; k += 32) jlist[dst + k] = src[k];
            continue;
        }
    }
    else
    {
        const uint32_t dst = jOffset[leaf], cnt = jOffset[leaf + 1] - dst, src = jOffsetPrev[leaf];
        if (jOffset[leaf + 1] > listCap)
        {
            if (lane == 0) atomicOr(err, int(kErrListFull));
            continue;
        }
        for (uint32_t k = lane; k < cnt; k += 32) jlist[dst + k] = jlistPrev[src + k];
        continue;
    }
    const int s = set[leaf];
    const int ns = setNodeStart[s], ne = setNodeStart[s + 1];
    const double4 ic = preCenter[leafPre[leaf]], is = preHalf[leafPre[leaf]];
    const double hmax = hm * setMargin[s];
    const double radHi = kRadKernel * hmax;
    const double ax = is.x + radHi, ay = is.y + radHi, az = is.z + radHi;
    const DevBox bx = boxes[s];
    const bool per = bx.periodic != 0;
    uint32_t count = 0, base = 0, cap = 0, stream = 0;
    if (Fill)
    {
        base = jOffset[leaf];
        cap = jOffset[leaf + 1] - base;
        if (jOffset[leaf + 1] > listCap)   // the preallocated list is too small: report, write nothing
        {
            if (lane == 0) atomicOr(err, int(kErrListFull));
            continue;
        }
    }
    const uint32_t lt = (1u << lane) - 1u;
    int p = ns;
    while (p < ne)
    {
        const int idx = p + lane;
        const bool valid = idx < ne;
        bool accept = false;
        int skip = 1, pl = -1;
        if (valid)
        {
            const double4 c = preCenter[idx];
            const double4 h = preHalf[idx];
            double d0 = fabs(ic.x - c.x), d1 = fabs(ic.y - c.y), d2 = fabs(ic.z - c.z);
            if (per)
            {
                d0 = fmin(d0, bx.len[0] - d0);
                d1 = fmin(d1, bx.len[1] - d1);
                d2 = fmin(d2, bx.len[2] - d2);
            }
            const double g0 = d0 - ax - h.x, g1 = d1 - ay - h.y, g2 = d2 - az - h.z;
            const double e0 = (g0 > 0.0) ? g0 : 0.0, e1 = (g1 > 0.0) ? g1 : 0.0, e2 = (g2 > 0.0) ? g2 : 0.0;
            accept = e0 * e0 + e1 * e1 + e2 * e2 <= 0.0;
            skip = preSkip[idx];
            pl = preLeaf[idx];
        }
        const uint32_t validMask = __ballot_sync(0xffffffffu, valid);
        const uint32_t rejMask = __ballot_sync(0xffffffffu, valid && !accept);
        int pos = 0;
        int next = p + 32;
        for (;;)
        {
            const uint32_t fromPos = (pos >= 32) ? 0u : (0xffffffffu << pos);
            const uint32_t rej = rejMask & fromPos;
            const int r = rej ? (__ffs(rej) - 1) : 32;
            const uint32_t runMask = validMask & fromPos & ((r >= 32) ? 0xffffffffu : ((1u << r) - 1u));
            const uint32_t emitMask = __ballot_sync(0xffffffffu, ((runMask >> lane) & 1u) && pl >= 0);
            if (Fill && ((emitMask >> lane) & 1u))
            {
                const uint32_t slot = count + __popc(emitMask & lt);
                if (slot < cap) jlist[base + slot] = pl;
                else atomicOr(err, int(kErrListCap));
            }
            if (!Fill && ((emitMask >> lane) & 1u))
            {
                stream += range[pl].y - range[pl].x;
                const uint32_t slot = count + __popc(emitMask & lt);
                if (slot < uint32_t(kWalkScratchB)) scratch[size_t(leaf) * kWalkScratchB + slot] = pl;
            }
            count += __popc(emitMask);
            if (r >= 32) { next = p + 32; break; }
            int rskip = __shfl_sync(0xffffffffu, skip, r);
            if (rskip < 1) rskip = 1;
            const int target = p + r + rskip;
            if (target >= p + 32 || target >= ne) { next = target; break; }
            pos = target - p;
        }
        p = next;
    }
    if (!Fill)
    {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) stream += __shfl_xor_sync(0xffffffffu, stream, o);
    }
    if (lane == 0)
    {
        if (Fill) { if (count != cap) atomicOr(err, int(kErrListCap)); }
        else
        {
            jcount[leaf] = count;
            jstream[leaf] = stream;
            listH[leaf] = hmax;
            walked[leaf] = 1;
        }
    }
    }
}

// Keep this walk's lists for the next one: counts, offsets and the used part of the list.
__global__ void keep_lists_kernel(int L, const uint32_t* __restrict__ jcount, const uint32_t* __restrict__ jOffset,
                                  const int* __restrict__ jlist, uint32_t listCap, uint32_t* __restrict__ jcountPrev,
                                  uint32_t* __restrict__ jOffsetPrev, int* __restrict__ jlistPrev)
{
    const long stride = long(gridDim.x) * blockDim.x;
    const long t0 = long(blockIdx.x) * blockDim.x + threadIdx.x;
    for (long t = t0; t < L; t += stride) jcountPrev[t] = jcount[t];
    for (long t = t0; t <= L; t += stride) jOffsetPrev[t] = jOffset[t];
    const long total = min(long(jOffset[L]), long(listCap));
    for (long t = t0; t < total; t += stride) jlistPrev[t] = jlist[t];
}

// Newton-Raphson step of one particle, FP64 (src/density_base.cu:294-333); returns
// whether it is still unconverged.
__device__ __forceinline__ bool nr_step_b(double rhoi, double gradhi, double hi, double pmass, double hfact,
                                          double tolh, double& rhoOut, double& gradOut, double& hOut, int& conv)
{
    const double hi1 = 1.0 / hi;
    const double hi31 = hi1 * hi1 * hi1;
    const double hi41 = hi31 * hi1;
    const double rho_i = rhoi * kCnormk * pmass * hi31;
    const double grad_i = gradhi * kCnormk * pmass * hi41;
    if (!(rho_i > 0.0))
    {
        rhoOut = 0.0; gradOut = 0.0; hOut = hi; conv = 0;
        return true;
    }
    const double rhoh_i = pmass * (hfact * hi1) * (hfact * hi1) * (hfact * hi1);
    const double funci = rhoh_i - rho_i;
    const double dhdrhoi = -hi / (3.0 * rhoh_i);
    const double omegai = 1.0 - dhdrhoi * grad_i;
    const double safe = (omegai > 0.0) ? omegai : fabs(omegai + 1e-300);
    const double hraw = hi - funci * dhdrhoi / safe;
    double hnew;
    if (hraw > 1.2 * hi) hnew = 1.2 * hi;
    else if (hraw < 0.8 * hi) hnew = 0.8 * hi;
    else hnew = hraw;
    rhoOut = rho_i; gradOut = grad_i; hOut = hnew;
    conv = (fabs((hnew - hi) / hi) < tolh) ? 1 : 0;
    return !conv;
}

// One Newton iteration (or, EvalAll, rho at the final h) over the work items of every
// set, taken dynamically by a persistent grid.  Each item carries its leaf; the leaf its
// set's mass, periodicity and box.  A cut item scans its set's tree for its own box
// instead of streaming the leaf's whole list.
template<bool Mixed, bool EvalAll, bool Staged>
__global__ void __launch_bounds__(kThreads, 5)   // 20 warps per SM (measured best of 4, 5, 6)
density_batch_kernel(const int4* __restrict__ items, int cap, const int* __restrict__ leafSet,
                     const uint2* __restrict__ range, const uint32_t* __restrict__ jOffset,
                     const uint32_t* __restrict__ jcount, const int* __restrict__ jlist, double4* __restrict__ xyzh,
                     double* __restrict__ rho, double* __restrict__ gradh, int* __restrict__ converged,
                     const double* __restrict__ pmassSet, double tolh, double hfact, const DevBox* __restrict__ boxes,
                     int* __restrict__ leafNext, int* __restrict__ nextLeaves, PreorderTree tree,
                     const int* __restrict__ setNodeStart, const int* __restrict__ leafPre,
                     const double* __restrict__ hmaxLeaf, DevScalars* __restrict__ ds, long long waitNs)
{
    __shared__ __align__(16) unsigned char sScr[kWarpsPerBlock][DensScratch<Mixed>::kBytes];
    __shared__ __align__(128) WarpStage sStage[Staged ? kWarpsPerBlock : 1];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    StageRef stage{nullptr, &ds->err, waitNs};
    if constexpr (Staged)
    {
        stage_init(sStage[wib]);
        stage.ws = &sStage[wib];
    }
    const int nHeavy = ds->itemsHeavy, nItems = nHeavy + ds->itemsLight;
    unsigned long long pairs = 0;
    for (;;)
    {
        const int w = next_item(ds, nHeavy, nItems, cap);
        if (w < 0) break;
        const int4 it = items[w];
        const int leaf = it.x;
        const Item d = decode_item(it, range[leaf].x);
        const int s = leafSet[leaf];
        const double pmass = pmassSet[s];
        const DevBox bxs = boxes[s];
        const bool per = bxs.periodic != 0;
        const int slot = group_slot(d.m0, d.m1, d.nAct, d.grp, d.G, lane);
        const bool mine = slot >= 0;
        const uint32_t i = d.g0 + uint32_t(mine ? slot : 0);
        const double4 pi = xyzh[i];
        double rhoi = 0.0, gradhi = 0.0;
        unsigned int gp = 0, gc = 0;
        auto src = list_source(jlist, jOffset[leaf], jcount[leaf], TableRanges{range}, xyzh);
        src.stage = stage;   // Staged: j ranges staged into shared memory by bulk copies
        if (w < nHeavy)
        {
            const double4 c = tree.center[leafPre[leaf]], h = tree.half[leafPre[leaf]];
            double hm = hmaxLeaf[leaf];
            if (!isfinite(hm) || hm <= 0.0) hm = 0.0;
            const double ext = kRadKernel * hm;
            src.walk = true;
            src.tree = tree;
            src.tree.n0 = setNodeStart[s];
            src.tree.n1 = setNodeStart[s + 1];
            src.rc = make_double3(c.x, c.y, c.z);
            src.re = make_double3(h.x + ext, h.y + ext, h.z + ext);
        }
        // one engine instance for open and periodic sets (zero periods fold nothing): half
        // the code the warps of a mixed ensemble would otherwise share the instruction
        // cache with
        density_group<true, Mixed, Staged, false>(sScr[wib], mine, d.ng, pi, per ? bxs.len[0] : 0.0, per ? bxs.len[1] : 0.0,
                                   per ? bxs.len[2] : 0.0, src, rhoi, gradhi, gp, gc);
        if (EvalAll)
        {
            // rho and d(rho)/dh at the converged h (src/density_base.cu:635-643)
            if (mine)
            {
                pairs += gp;
                const double hi1 = 1.0 / pi.w;
                const double hi31 = hi1 * hi1 * hi1;
                rho[i] = rhoi * kCnormk * pmass * hi31;
                gradh[i] = gradhi * kCnormk * pmass * (hi31 * hi1);
            }
            continue;
        }
        bool still = false;
        if (mine)
        {
            pairs += gp;
            double ro, go, ho;
            int conv;
            still = nr_step_b(rhoi, gradhi, pi.w, pmass, hfact, tolh, ro, go, ho, conv);
            rho[i] = ro;
            gradh[i] = go;
            reinterpret_cast<double*>(xyzh + i)[3] = ho;
            converged[i] = conv;
        }
        const uint32_t stillMask = __ballot_sync(0xffffffffu, still);
        if (stillMask && lane == 0)
        {
            atomicAdd(&ds->unconverged, __popc(stillMask));
            if (atomicExch(&leafNext[leaf], 1) == 0) nextLeaves[atomicAdd(&ds->nextActive, 1)] = leaf;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    if (lane == 0) atomicAdd(&ds->pairs[0], pairs);
}

__global__ void copy_active_kernel(const int* __restrict__ src, int* __restrict__ dst, const DevScalars* __restrict__ ds,
                                   int cap)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < cap && t < ds->nextActive) dst[t] = src[t];
}

// End of one Newton iteration: record it, adopt the next active set, and decide
// whether the loop goes on (the graph's while condition when run as a graph).
__global__ void loop_epilogue_kernel(LoopState* ls, const DevScalars* ds, cudaGraphConditionalHandle handle,
                                     int setCondition)
{
    if (ls->iter < 128) ls->activePerIter[ls->iter] = ls->nActiveParticles;
    ls->iter += 1;
    ls->nActiveLeaves = ds->nextActive;
    ls->nActiveParticles = ds->unconverged;
    const int more = (ls->nActiveParticles > 0 && ls->iter < ls->maxIter && ds->err == 0) ? 1 : 0;
    if (setCondition) cudaGraphSetConditional(handle, more);
}

__global__ void iota_kernel_b(int* __restrict__ a, int n)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) a[i] = int(i);
}

__global__ void scatter_kernel_b(const int* __restrict__ order, int n, const double4* __restrict__ xyzh,
                                 const double* __restrict__ rho, const double* __restrict__ gradh, double* __restrict__ out)
{
    const long k = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int o = order[k];
    out[o] = xyzh[k].w;
    out[size_t(n) + o] = rho[k];
    out[2 * size_t(n) + o] = gradh[k];
}

} // namespace

// ====================================================================== host side
static void batch_build(Batch& B)
{
    State& s = B.core;
    const int n = B.n, ns = B.nsets;
    DevScalars* ds = s.dscal.get();
    cudaEvent_t e0 = ev(s);
    set_box_kernel_b<<<ns, 256, 0, s.st>>>(B.dOffs.get(), B.setPer.get(), B.setBox6.get(), B.ux.get(), B.uy.get(),
                                           B.uz.get(), B.boxes.get());
    COSMO_LAUNCHED();
    keys_kernel_b<<<iceil(n, kBlk), kBlk, 0, s.st>>>(B.ux.get(), B.uy.get(), B.uz.get(), B.uh.get(), B.setOf.get(), n,
                                                    B.boxes.get(), B.keysA.get());
    COSMO_LAUNCHED();
    // stable key sort (8 passes), then stable set-id passes: (set, key) order
    radix_sort_u64(s, B.keysA.get(), B.keysB.get(), B.orderA.get(), B.orderB.get(), n, true);
    uint64_t* kA = B.keysA.get(); uint64_t* kB = B.keysB.get();
    int* vA = B.orderA.get(); int* vB = B.orderB.get();
    const int setPasses = ns <= 1 ? 0 : (ns <= 256 ? 1 : 2);
    if (setPasses)
    {
        const int tiles = iceil(n, kSortTile);
        s.sortLookback.resize(size_t(setPasses) * tiles * 256, s.st);
        COSMO_CUDA(cudaMemsetAsync(s.sortLookback.get(), 0, size_t(setPasses) * tiles * 256 * 4, s.st));
        COSMO_CUDA(cudaMemsetAsync(&ds->sortTiles[8], 0, 2 * sizeof(unsigned int), s.st));
        B.setHist.resize(512, s.st);
        B.setBase.resize(512, s.st);
        COSMO_CUDA(cudaMemsetAsync(B.setHist.get(), 0, 512 * 4, s.st));
        for (int p = 0; p < setPasses; ++p)
        {
            set_hist_kernel<<<std::min(iceil(n, kBlk), 2 * s.numSMs), kBlk, 0, s.st>>>(B.setOf.get(), n, 8 * p,
                                                                                      B.setHist.get() + 256 * p);
            COSMO_LAUNCHED();
        }
        digit_base_kernel<<<setPasses, 256, 0, s.st>>>(B.setHist.get(), B.setBase.get());
        COSMO_LAUNCHED();
        for (int p = 0; p < setPasses; ++p)
        {
            onesweep_set_kernel<<<tiles, kSortThreads, 0, s.st>>>(kA, vA, kB, vB, n, 8 * p, B.setBase.get() + 256 * p,
                                                                 s.sortLookback.get() + size_t(p) * tiles * 256,
                                                                 &ds->sortTiles[8 + p], &ds->err, B.setOf.get(),
                                                                 wait_limit_ns());
            COSMO_LAUNCHED();
            std::swap(kA, kB);
            std::swap(vA, vB);
        }
        if (kA != B.keysA.get())
        {
            COSMO_CUDA(cudaMemcpyAsync(B.keysA.get(), kA, size_t(n) * 8, cudaMemcpyDeviceToDevice, s.st));
            COSMO_CUDA(cudaMemcpyAsync(B.orderA.get(), vA, size_t(n) * 4, cudaMemcpyDeviceToDevice, s.st));
        }
    }
    COSMO_CUDA(cudaMemsetAsync(B.nAliveSet.get(), 0, size_t(ns) * 4, s.st));
    alive_kernel_b<<<iceil(n, kBlk), kBlk, 0, s.st>>>(B.keysA.get(), B.dOffs.get(), ns, n, B.nAliveSet.get());
    COSMO_LAUNCHED();
    gather_kernel_b<<<iceil(n, kBlk), kBlk, 0, s.st>>>(B.orderA.get(), n, B.ux.get(), B.uy.get(), B.uz.get(),
                                                       B.uh.get(), B.xyzh.get());
    COSMO_LAUNCHED();

    // forest leaves: one root per set, split while a node holds more than its bucket
    int L = ns;
    B.leafKey.resize(L, s.st);
    B.leafSet.resize(L, s.st);
    roots_kernel<<<iceil(ns, 256), 256, 0, s.st>>>(ns, B.leafKey.get(), B.leafSet.get());
    COSMO_LAUNCHED();
    for (int round = 0; round < 64; ++round)
    {
        B.ops.resize(L, s.st);
        B.opsScan.resize(size_t(L) + 1, s.st);
        B.leafRange.resize(L, s.st);
        leaf_count_kernel_b<<<iceil(L, kBlk), kBlk, 0, s.st>>>(B.leafKey.get(), B.leafSet.get(), L, B.keysA.get(),
                                                              B.dOffs.get(), B.nAliveSet.get(), B.bucket.get(),
                                                              B.ops.get(), B.leafRange.get());
        COSMO_LAUNCHED();
        const int total = int(scan_exclusive(s, B.ops.get(), B.opsScan.get(), L, true));
        if (total == L) break;
        B.leafKey2.resize(total, s.st);
        B.leafSet2.resize(total, s.st);
        leaf_split_kernel_b<<<iceil(L, kBlk), kBlk, 0, s.st>>>(B.leafKey.get(), B.leafSet.get(), L, B.ops.get(),
                                                              B.opsScan.get(), B.leafKey2.get(), B.leafSet2.get());
        COSMO_LAUNCHED();
        std::swap(B.leafKey, B.leafKey2);
        std::swap(B.leafSet, B.leafSet2);
        L = total;
    }
    B.nLeaves = L;
    B.setLeafStart.resize(size_t(ns) + 1, s.st);
    set_leaf_start_kernel<<<iceil(L + 1, kBlk), kBlk, 0, s.st>>>(B.leafSet.get(), L, ns, B.setLeafStart.get());
    COSMO_LAUNCHED();
    B.nodeCount.resize(L, s.st);
    B.leafPreStart.resize(size_t(L) + 1, s.st);
    node_count_kernel_b<<<iceil(L, kBlk), kBlk, 0, s.st>>>(B.leafKey.get(), B.leafSet.get(), L, B.nodeCount.get());
    COSMO_LAUNCHED();
    const int numNodes = int(scan_exclusive(s, B.nodeCount.get(), B.leafPreStart.get(), L, true));
    B.numNodes = numNodes;
    B.setNodeStart.resize(size_t(ns) + 1, s.st);
    set_node_start_kernel<<<iceil(ns + 1, 256), 256, 0, s.st>>>(B.setLeafStart.get(), B.leafPreStart.get(), ns,
                                                                B.setNodeStart.get());
    COSMO_LAUNCHED();
    for (auto* b : {&B.preLeaf, &B.preSkip}) b->resize(numNodes, s.st);
    B.preCenter.resize(numNodes, s.st);
    B.preHalf.resize(numNodes, s.st);
    B.leafPre.resize(L, s.st);
    node_emit_kernel_b<<<iceil(L, kBlk), kBlk, 0, s.st>>>(B.leafKey.get(), B.leafSet.get(), L, B.leafPreStart.get(),
                                                         B.setLeafStart.get(), B.setNodeStart.get(), B.boxes.get(),
                                                         B.preLeaf.get(), B.preSkip.get(), B.leafPre.get(),
                                                         B.preCenter.get(), B.preHalf.get());
    COSMO_LAUNCHED();
    B.hmaxLeaf.resize(L, s.st);
    B.jcount.resize(L, s.st);
    B.jstream.resize(L, s.st);
    B.jcountPrev.resize(L, s.st);
    B.jOffsetPrev.resize(size_t(L) + 1, s.st);
    B.walked.resize(L, s.st);
    B.walkScratch.resize(size_t(L) * kWalkScratchB, s.st);
    B.listH.resize(L, s.st);
    B.leafNext.resize(L, s.st);
    B.items.resize(std::max(B.n, 1), s.st);
    B.jOffset.resize(size_t(L) + 1, s.st);
    B.activeA.resize(L, s.st);
    B.activeB.resize(L, s.st);
    B.allLeaves.resize(L, s.st);
    iota_kernel_b<<<iceil(L, kBlk), kBlk, 0, s.st>>>(B.activeA.get(), L);
    COSMO_LAUNCHED();
    iota_kernel_b<<<iceil(L, kBlk), kBlk, 0, s.st>>>(B.allLeaves.get(), L);
    COSMO_LAUNCHED();
    cudaEvent_t e1 = ev(s);
    read_scalars(s);
    B.tBuild = elapsed_s(e0, e1);
}

// The gather lists of the given leaves (count on the device): a leaf whose kept list
// still covers its hmax copies it, the others walk (the count pass keeps what it walks
// for the fill pass).  The counts of all other leaves are zero, so the scan sizes the
// list storage for these leaves only.
static void walk_lists(Batch& B, bool fill, const int* leaves, const int* countPtr)
{
    State& s = B.core;
    const int L = B.nLeaves;
    if (!fill) COSMO_CUDA(cudaMemsetAsync(B.jcount.get(), 0, size_t(L) * sizeof(uint32_t), s.st));
    const int blocks = std::max(1, std::min(iceil(long(L) * 32, 256), 16 * s.numSMs));
    auto go = [&](auto kern) {
        kern<<<blocks, 256, 0, s.st>>>(leaves, countPtr, B.leafSet.get(), B.setNodeStart.get(), B.leafPre.get(),
                                       B.hmaxLeaf.get(),
                                       B.preCenter.get(), B.preHalf.get(), B.preSkip.get(), B.preLeaf.get(),
                                       B.boxes.get(), B.jcount.get(), B.jOffset.get(), B.jlist.get(), B.listCap,
                                       &s.dscal.get()->err, B.leafRange.get(), B.jstream.get(), B.listH.get(),
                                       B.walked.get(), B.jcountPrev.get(), B.jOffsetPrev.get(), B.jlistPrev.get(),
                                       B.setMargin.get(), B.walkScratch.get());
    };
    if (fill) go(list_walk_kernel_b<true>);
    else go(list_walk_kernel_b<false>);
    COSMO_LAUNCHED();
}

// Keep the lists just filled (all leaves) as the source the next walk copies from.
static void keep_lists(Batch& B)
{
    State& s = B.core;
    const int L = B.nLeaves;
    keep_lists_kernel<<<4 * s.numSMs, 256, 0, s.st>>>(L, B.jcount.get(), B.jOffset.get(), B.jlist.get(), B.listCap,
                                                     B.jcountPrev.get(), B.jOffsetPrev.get(), B.jlistPrev.get());
    COSMO_LAUNCHED();
}

// Work items of the given leaves (count on the device), then the density kernel over
// them: a Newton iteration, or (evalAll) rho at the final h of every live particle.
static void run_items(Batch& B, const int* leaves, const int* countPtr, bool evalAll, double tolh, double hfact)
{
    State& s = B.core;
    DevScalars* ds = s.dscal.get();
    const int L = B.nLeaves;
    const int cap = std::max(B.n, 1);
    begin_iteration_kernel<<<std::min(iceil(L, 256), 4 * s.numSMs), 256, 0, s.st>>>(ds, B.leafNext.get(), L);
    COSMO_LAUNCHED();
    plan_items_table_kernel<<<s.numSMs * 8, kThreads, 0, s.st>>>(leaves, countPtr, B.leafRange.get(),
                                                                  evalAll ? nullptr : B.converged.get(),
                                                                  B.jstream.get(), B.xyzh.get(), B.items.get(), cap,
                                                                  ds, B.leafSet.get(), B.setSplit.get());
    COSMO_LAUNCHED();
    const PreorderTree tree{B.preCenter.get(), B.preHalf.get(), B.preSkip.get(), B.preLeaf.get(), 0, 0};
    auto go = [&](auto kern) {
        kern<<<persistent_grid(s, kern, kThreads), kThreads, 0, s.st>>>(
            B.items.get(), cap, B.leafSet.get(), B.leafRange.get(), B.jOffset.get(), B.jcount.get(), B.jlist.get(),
            B.xyzh.get(), B.rho.get(), B.gradh.get(), B.converged.get(), B.pmass.get(), tolh, hfact, B.boxes.get(),
            B.leafNext.get(), B.activeB.get(), tree, B.setNodeStart.get(), B.leafPre.get(), B.hmaxLeaf.get(), ds,
            wait_limit_ns());
    };
    const bool mx = s.precision == 1, st = s.staging != 0;
    if (evalAll)
    {
        if (mx) st ? go(density_batch_kernel<true, true, true>) : go(density_batch_kernel<true, true, false>);
        else st ? go(density_batch_kernel<false, true, true>) : go(density_batch_kernel<false, true, false>);
    }
    else
    {
        if (mx) st ? go(density_batch_kernel<true, false, true>) : go(density_batch_kernel<true, false, false>);
        else st ? go(density_batch_kernel<false, false, true>) : go(density_batch_kernel<false, false, false>);
    }
    COSMO_LAUNCHED();
}

// One Newton-Raphson iteration, every count read on the device: hmax of the active
// leaves, the gather lists of all leaves (count, scan, fill: a leaf whose hmax is still
// inside the radius its kept list was walked at copies that list, the others walk), the
// density kernel over the active leaves of all sets, the lists kept for the next
// iteration, the new active set, and the loop bookkeeping.  Run eagerly, or captured
// once as the body of a graph's while node.
static void nr_iteration(Batch& B, double tolh, double hfact, cudaGraphConditionalHandle handle, int setCond)
{
    State& s = B.core;
    DevScalars* ds = s.dscal.get();
    LoopState* ls = B.loop.get();
    const int L = B.nLeaves;
    hmax_leaf_kernel_b<<<iceil(L, 256), 256, 0, s.st>>>(B.xyzh.get(), B.leafRange.get(), B.activeA.get(),
                                                       &ls->nActiveLeaves, B.hmaxLeaf.get());
    COSMO_LAUNCHED();
    walk_lists(B, false, B.allLeaves.get(), &ls->nAll);
    scan_exclusive(s, B.jcount.get(), B.jOffset.get(), L, false);
    walk_lists(B, true, B.allLeaves.get(), &ls->nAll);
    run_items(B, B.activeA.get(), &ls->nActiveLeaves, false, tolh, hfact);
    keep_lists(B);
    copy_active_kernel<<<iceil(L, 256), 256, 0, s.st>>>(B.activeB.get(), B.activeA.get(), ds, L);
    COSMO_LAUNCHED();
    loop_epilogue_kernel<<<1, 1, 0, s.st>>>(ls, ds, handle, setCond);
    COSMO_LAUNCHED();
}

// rho and d(rho)/dh of every live particle at its final h (one more gather pass).
static void final_rho(Batch& B)
{
    State& s = B.core;
    DevScalars* ds = s.dscal.get();
    LoopState* ls = B.loop.get();
    const int L = B.nLeaves;
    hmax_leaf_kernel_b<<<iceil(L, 256), 256, 0, s.st>>>(B.xyzh.get(), B.leafRange.get(), B.allLeaves.get(), &ls->nAll,
                                                       B.hmaxLeaf.get());
    COSMO_LAUNCHED();
    walk_lists(B, false, B.allLeaves.get(), &ls->nAll);
    const uint32_t total = scan_exclusive(s, B.jcount.get(), B.jOffset.get(), L, true);
    if (total > B.listCap)
    {
        B.listCap = total + total / 4 + 1024;
        B.jlist.resize(B.listCap, s.st);   // the kept lists (jlistPrev) stay where they are
    }
    walk_lists(B, true, B.allLeaves.get(), &ls->nAll);
    run_items(B, B.allLeaves.get(), &ls->nAll, true, 0.0, 0.0);
}

static int batch_solve(Batch& B, double tolh, double hfact, int maxIter, int flags, int attempt = 0)
{
    State& s = B.core;
    if (!(hfact > 0.0)) hfact = kHfactDefault;
    maxIter = std::max(1, std::min(maxIter, 128));
    ev_reset(s);
    DevScalars* ds = s.dscal.get();
    COSMO_CUDA(cudaMemsetAsync(B.rho.get(), 0, size_t(B.n) * 8, s.st));
    COSMO_CUDA(cudaMemsetAsync(B.gradh.get(), 0, size_t(B.n) * 8, s.st));
    COSMO_CUDA(cudaMemsetAsync(B.converged.get(), 0, size_t(B.n) * 4, s.st));
    COSMO_CUDA(cudaMemsetAsync(&ds->pairs[0], 0, sizeof(ds->pairs), s.st));
    cudaEvent_t t0 = ev(s);
    batch_build(B);
    const int L = B.nLeaves;
    long long nAliveTotal = 0;
    {
        std::vector<int> na(B.nsets);
        COSMO_CUDA(cudaMemcpyAsync(na.data(), B.nAliveSet.get(), size_t(B.nsets) * 4, cudaMemcpyDeviceToHost, s.st));
        COSMO_CUDA(cudaStreamSynchronize(s.st));
        for (int v : na) nAliveTotal += v;
    }
    B.loop.resize(1, s.st);
    LoopState init{};
    init.nActiveLeaves = L;
    init.nActiveParticles = int(nAliveTotal);
    init.iter = 0;
    init.maxIter = maxIter;
    init.nAll = L;
    COSMO_CUDA(cudaMemcpyAsync(B.loop.get(), &init, sizeof(LoopState), cudaMemcpyHostToDevice, s.st));
    // Size the list storage from the first iteration's lists (lists grow with h; a build
    // that outgrows the storage reports it and the solve is repeated with twice as much),
    // then fill and keep them: the first iteration copies them.
    COSMO_CUDA(cudaMemsetAsync(B.jcountPrev.get(), 0, size_t(L) * sizeof(uint32_t), s.st));
    hmax_leaf_kernel_b<<<iceil(L, 256), 256, 0, s.st>>>(B.xyzh.get(), B.leafRange.get(), B.activeA.get(),
                                                       &B.loop.get()->nActiveLeaves, B.hmaxLeaf.get());
    COSMO_LAUNCHED();
    walk_lists(B, false, B.activeA.get(), &B.loop.get()->nActiveLeaves);
    const uint32_t total0 = scan_exclusive(s, B.jcount.get(), B.jOffset.get(), L, true);
    const uint32_t want = (total0 << (1 + attempt)) + 1024;
    if (B.listCap < want) B.listCap = want;
    B.jlist.resize(B.listCap, s.st);
    B.jlistPrev.resize(B.listCap, s.st);
    s.scanTmp.resize(size_t(iceil(L, 4096)) + 1, s.st);
    walk_lists(B, true, B.activeA.get(), &B.loop.get()->nActiveLeaves);
    keep_lists(B);
    COSMO_CUDA(cudaStreamSynchronize(s.st));
    cudaEvent_t t1 = ev(s);

    const bool useGraph = (flags & COSMO_BATCH_GRAPH) != 0;
    B.graphUsed = useGraph;
    if (useGraph)
    {
        cudaGraph_t graph = nullptr;
        COSMO_CUDA(cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle handle;
        COSMO_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        COSMO_CUDA(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        COSMO_CUDA(cudaStreamBeginCaptureToGraph(s.st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        nr_iteration(B, tolh, hfact, handle, 1);
        COSMO_CUDA(cudaStreamEndCapture(s.st, &body));
        cudaGraphExec_t exec = nullptr;
        COSMO_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        COSMO_CUDA(cudaGraphLaunch(exec, s.st));
        COSMO_CUDA(cudaStreamSynchronize(s.st));
        COSMO_CUDA(cudaGraphExecDestroy(exec));
        COSMO_CUDA(cudaGraphDestroy(graph));
    }
    else
    {
        LoopState h{};
        for (int iter = 0; iter < maxIter; ++iter)
        {
            nr_iteration(B, tolh, hfact, cudaGraphConditionalHandle(0), 0);
            COSMO_CUDA(cudaMemcpyAsync(&h, B.loop.get(), 16, cudaMemcpyDeviceToHost, s.st));
            COSMO_CUDA(cudaStreamSynchronize(s.st));
            if (h.nActiveParticles == 0) break;
            read_scalars(s);
            if (s.hscal->err) break;
        }
    }
    cudaEvent_t t2 = ev(s);
    read_scalars(s);
    if ((s.hscal->err & kErrListFull) && attempt < 6)
    {
        COSMO_CUDA(cudaMemsetAsync(&ds->err, 0, sizeof(int), s.st));
        return batch_solve(B, tolh, hfact, maxIter, flags, attempt + 1);
    }
    LoopState fin{};
    COSMO_CUDA(cudaMemcpyAsync(&fin, B.loop.get(), sizeof(LoopState), cudaMemcpyDeviceToHost, s.st));
    COSMO_CUDA(cudaStreamSynchronize(s.st));
    B.itersRun = fin.iter;
    B.unconverged = fin.nActiveParticles;
    B.activePerIter.assign(fin.activePerIter, fin.activePerIter + std::min(fin.iter, 128));
    if (flags & COSMO_BATCH_FINAL_RHO) final_rho(B);
    cudaEvent_t t3 = ev(s);
    check_dev_err(s, "cosmo_batch_density");
    B.tBuild = elapsed_s(t0, t1);
    B.tNR = elapsed_s(t1, t2);
    B.tList = 0.0;
    B.tTotal = elapsed_s(t0, t3);
    B.pairs = s.hscal->pairs[0];
    return B.unconverged > 0 ? 1 : 0;
}

} // namespace cosmo

using namespace cosmo;

extern "C" {

int cosmo_batch_init(int nsets, const int* offsets)
{
    if (nsets < 1 || offsets == nullptr || offsets[0] != 0) return -1;
    for (int s = 0; s < nsets; ++s)
        if (offsets[s + 1] < offsets[s]) return -1;
    Batch& B = batch();
    State& s = B.core;
    ensure_init(s);
    const int n = offsets[nsets];
    if (n < 1) return -1;
    B.nsets = nsets;
    B.n = n;
    B.offs.assign(offsets, offsets + nsets + 1);
    for (auto* b : {&B.dOffs, &B.setLeafStart, &B.setNodeStart}) b->resize(size_t(nsets) + 1, s.st);
    for (auto* b : {&B.nAliveSet, &B.bucket, &B.setPer}) b->resize(nsets, s.st);
    B.pmass.resize(nsets, s.st);
    B.setBox6.resize(size_t(6) * nsets, s.st);
    B.boxes.resize(nsets, s.st);
    for (auto* b : {&B.ux, &B.uy, &B.uz, &B.uh, &B.rho, &B.gradh}) b->resize(n, s.st);
    B.xyzh.resize(n, s.st);
    for (auto* b : {&B.converged, &B.orderA, &B.orderB, &B.setOf}) b->resize(n, s.st);
    B.keysA.resize(n, s.st);
    B.keysB.resize(n, s.st);
    s.xfer.resize(size_t(3) * n, s.st);
    COSMO_CUDA(cudaMemcpyAsync(B.dOffs.get(), offsets, size_t(nsets + 1) * 4, cudaMemcpyHostToDevice, s.st));
    setof_kernel<<<iceil(n, 256), 256, 0, s.st>>>(B.dOffs.get(), nsets, n, B.setOf.get());
    COSMO_LAUNCHED();
    std::vector<int> bucket(nsets, int(kBucket)), per(nsets, 0);
    COSMO_CUDA(cudaMemcpyAsync(B.bucket.get(), bucket.data(), size_t(nsets) * 4, cudaMemcpyHostToDevice, s.st));
    B.setMargin.resize(nsets, s.st);
    B.setSplit.resize(nsets, s.st);
    std::vector<double> margin(nsets, kBatchListMargin);
    std::vector<uint2> split(nsets, make_uint2(kSplitStream, kSplitWork));
    COSMO_CUDA(cudaMemcpyAsync(B.setMargin.get(), margin.data(), size_t(nsets) * 8, cudaMemcpyHostToDevice, s.st));
    COSMO_CUDA(cudaMemcpyAsync(B.setSplit.get(), split.data(), size_t(nsets) * 8, cudaMemcpyHostToDevice, s.st));
    B.tuning.assign(size_t(nsets) * 4, 0.0);
    for (int k = 0; k < nsets; ++k)
    {
        B.tuning[4 * k] = kBucket;
        B.tuning[4 * k + 1] = kBatchListMargin;
        B.tuning[4 * k + 2] = kSplitStream;
        B.tuning[4 * k + 3] = kSplitWork;
    }
    COSMO_CUDA(cudaMemcpyAsync(B.setPer.get(), per.data(), size_t(nsets) * 4, cudaMemcpyHostToDevice, s.st));
    COSMO_CUDA(cudaStreamSynchronize(s.st));
    return 0;
}

void cosmo_batch_set_params(const double* pmass, const int* periodic, const double* box6)
{
    Batch& B = batch();
    State& s = B.core;
    const int ns = B.nsets;
    COSMO_CUDA(cudaMemcpyAsync(B.pmass.get(), pmass, size_t(ns) * 8, cudaMemcpyHostToDevice, s.st));
    std::vector<int> per(ns, 0);
    std::vector<double> bx(size_t(6) * ns, 0.0);
    if (periodic) std::copy(periodic, periodic + ns, per.begin());
    if (box6) std::copy(box6, box6 + 6 * size_t(ns), bx.begin());
    COSMO_CUDA(cudaMemcpyAsync(B.setPer.get(), per.data(), size_t(ns) * 4, cudaMemcpyHostToDevice, s.st));
    COSMO_CUDA(cudaMemcpyAsync(B.setBox6.get(), bx.data(), size_t(6) * ns * 8, cudaMemcpyHostToDevice, s.st));
    COSMO_CUDA(cudaStreamSynchronize(s.st));
}

void cosmo_batch_set_bucket(const int* bucketPerSet)
{
    Batch& B = batch();
    State& s = B.core;
    COSMO_CUDA(cudaMemcpyAsync(B.bucket.get(), bucketPerSet, size_t(B.nsets) * 4, cudaMemcpyHostToDevice, s.st));
    COSMO_CUDA(cudaStreamSynchronize(s.st));
    for (int k = 0; k < B.nsets; ++k) B.tuning[4 * size_t(k)] = bucketPerSet[k];
}

void cosmo_batch_set_staging(int on)
{
    Batch& B = batch();
    ensure_init(B.core);
    B.core.staging = on != 0 ? 1 : 0;
}

int cosmo_batch_set_tuning(const int* bucket, const double* listMargin, const int* splitStream, const int* splitWork)
{
    Batch& B = batch();
    State& s = B.core;
    const int ns = B.nsets;
    if (ns < 1) return -1;
    for (int k = 0; k < ns; ++k)
    {
        if (bucket && (bucket[k] < kMinTuneBucket || bucket[k] > kMaxTuneBucket)) return -1;
        if (listMargin && !(listMargin[k] >= 1.0 && listMargin[k] <= 2.0)) return -1;
        if (splitStream && splitStream[k] < 32) return -1;
        if (splitWork && splitWork[k] < 32) return -1;
    }
    std::vector<double> margin(ns);
    std::vector<uint2> split(ns);
    for (int k = 0; k < ns; ++k)
    {
        double* t = &B.tuning[4 * size_t(k)];
        if (bucket) t[0] = bucket[k];
        if (listMargin) t[1] = listMargin[k];
        if (splitStream) t[2] = splitStream[k];
        if (splitWork) t[3] = splitWork[k];
        margin[k] = t[1];
        split[k] = make_uint2(uint32_t(t[2]), uint32_t(t[3]));
    }
    std::vector<int> bk(ns);
    for (int k = 0; k < ns; ++k) bk[k] = int(B.tuning[4 * size_t(k)]);
    COSMO_CUDA(cudaMemcpyAsync(B.bucket.get(), bk.data(), size_t(ns) * 4, cudaMemcpyHostToDevice, s.st));
    COSMO_CUDA(cudaMemcpyAsync(B.setMargin.get(), margin.data(), size_t(ns) * 8, cudaMemcpyHostToDevice, s.st));
    COSMO_CUDA(cudaMemcpyAsync(B.setSplit.get(), split.data(), size_t(ns) * 8, cudaMemcpyHostToDevice, s.st));
    COSMO_CUDA(cudaStreamSynchronize(s.st));
    return 0;
}

void cosmo_batch_upload(const double* x, const double* y, const double* z, const double* h)
{
    Batch& B = batch();
    State& s = B.core;
    if (B.n < 1) return;   // no batch initialised: nothing to receive
    const size_t bytes = size_t(B.n) * 8;
    COSMO_CUDA(cudaMemcpyAsync(B.ux.get(), x, bytes, cudaMemcpyHostToDevice, s.st));
    COSMO_CUDA(cudaMemcpyAsync(B.uy.get(), y, bytes, cudaMemcpyHostToDevice, s.st));
    COSMO_CUDA(cudaMemcpyAsync(B.uz.get(), z, bytes, cudaMemcpyHostToDevice, s.st));
    COSMO_CUDA(cudaMemcpyAsync(B.uh.get(), h, bytes, cudaMemcpyHostToDevice, s.st));
    COSMO_CUDA(cudaStreamSynchronize(s.st));
}

int cosmo_batch_density(double tolh, double hfact, int maxIter, int flags)
{
    Batch& B = batch();
    if (B.n < 1) return -1;
    B.core.precision = state().precision;
    return batch_solve(B, tolh, hfact, maxIter > 0 ? maxIter : 100, flags);
}

void cosmo_batch_download(double* h, double* rho, double* gradh)
{
    Batch& B = batch();
    State& s = B.core;
    const int n = B.n;
    if (n < 1) return;   // no batch initialised: nothing to send
    scatter_kernel_b<<<iceil(n, 256), 256, 0, s.st>>>(B.orderA.get(), n, B.xyzh.get(), B.rho.get(), B.gradh.get(),
                                                     s.xfer.get());
    COSMO_LAUNCHED();
    const size_t bytes = size_t(n) * 8;
    COSMO_CUDA(cudaMemcpyAsync(h, s.xfer.get(), bytes, cudaMemcpyDeviceToHost, s.st));
    COSMO_CUDA(cudaMemcpyAsync(rho, s.xfer.get() + n, bytes, cudaMemcpyDeviceToHost, s.st));
    COSMO_CUDA(cudaMemcpyAsync(gradh, s.xfer.get() + 2 * size_t(n), bytes, cudaMemcpyDeviceToHost, s.st));
    COSMO_CUDA(cudaStreamSynchronize(s.st));
}

double cosmo_batch_scalar(const char* name)
{
    Batch& B = batch();
    const std::string k(name);
    if (k == "nLeaves") return B.nLeaves;
    if (k == "numNodes") return B.numNodes;
    if (k == "itersRun") return B.itersRun;
    if (k == "unconverged") return B.unconverged;
    if (k == "pairs") return double(B.pairs);
    if (k == "updates")
    {
        long long u = 0;
        for (long long v : B.activePerIter) u += v;
        return double(u);
    }
    if (k == "t_build") return B.tBuild;
    if (k == "t_total") return B.tTotal;
    if (k == "t_nr") return B.tNR;
    if (k == "graph") return B.graphUsed ? 1.0 : 0.0;
    if (k == "t_nr") return B.tNR;
    if (k == "t_list") return B.tList;
    return NAN;
}

} // extern "C"
