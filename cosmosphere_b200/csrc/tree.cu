/*
 * tree.cu -- Hilbert keys, the onesweep radix sort, the cornerstone leaf tree, the linked
 * octree with node geometry, hmax, and the j-leaf list walk.  The B200 counterpart of the
 * reference's src/tree.cu and include/tree.cuh, written without Thrust or Cornerstone.
 *
 * Parity notes (the oracle restates the same definitions):
 *   keys     21-bit quantisation of (x - lo) * 2^21/len, Skilling's Hilbert curve;
 *            h <= 0 (or NaN) gives ~0, which sorts last (include/tree.cuh:89-105).
 *   sort     stable LSD radix sort of (key, index): the order is the unique stable one.
 *   leaves   split from the root while a node holds more than 64 particles (a level-21
 *            node never splits): the fixed point of src/tree.cu:126-136 from its seed.
 *   octree   BFS order = placeholder prefixes sorted, as Cornerstone's OctreeData;
 *            childOffsets 0 marks a leaf, internalToLeaf is -1 for internal nodes.
 *   lists    the reference's accept tests (include/tree.cuh:228-252); leaves emitted in
 *            ascending order by a stackless pre-order scan (no stack, nothing dropped).
 */
#include <algorithm>

#include "sort.cuh"
#include "state.hpp"

namespace cosmo {

namespace {

// ------------------------------------------------------------------ bbox and keys
__global__ void bbox_partial_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                    const double* __restrict__ z, int n, double* __restrict__ part)
{
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
    {
        const double c[3] = {x[i], y[i], z[i]};
#pragma unroll
        for (int d = 0; d < 3; ++d) { mn[d] = fmin(mn[d], c[d]); mx[d] = fmax(mx[d], c[d]); }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
            mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
    __shared__ double s[8][6];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int d = 0; d < 3; ++d) { s[warp][d] = mn[d]; s[warp][3 + d] = mx[d]; }
    __syncthreads();
    if (threadIdx.x < 6)
    {
        const int c = threadIdx.x;
        double v = s[0][c];
        for (int w = 1; w < int(blockDim.x >> 5); ++w) v = (c < 3) ? fmin(v, s[w][c]) : fmax(v, s[w][c]);
        part[blockIdx.x * 6 + c] = v;
    }
}

// Open boundaries (src/tree.cu:54-72): a cube of side 1.00001 x the largest span,
// centred on the particles.
// One block partial holding given extents (min x, y, z then max x, y, z).
__global__ void set_extent_kernel(double* part, double x0, double x1, double y0, double y1, double z0, double z1)
{
    if (threadIdx.x != 0) return;
    part[0] = x0; part[1] = y0; part[2] = z0;
    part[3] = x1; part[4] = y1; part[5] = z1;
}

__global__ void bbox_final_kernel(const double* __restrict__ part, int nb, DevBox* box)
{
    // one warp: lanes stride over the block partials, then a shuffle reduction (min and
    // max are exact, so any order gives the serial result)
    const int lane = threadIdx.x & 31;
    if (threadIdx.x >= 32) return;
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int b = lane; b < nb; b += 32)
        for (int d = 0; d < 3; ++d) { mn[d] = fmin(mn[d], part[6 * b + d]); mx[d] = fmax(mx[d], part[6 * b + 3 + d]); }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        for (int d = 0; d < 3; ++d)
        {
            mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
            mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
    if (lane != 0) return;
    const double sx = mx[0] - mn[0], sy = mx[1] - mn[1], sz = mx[2] - mn[2];
    double span = (sx < sy) ? sy : sx;
    span = (span < sz) ? sz : span;
    span = span * 1.00001;
    const double half = 0.5 * span;
    DevBox b;
    for (int d = 0; d < 3; ++d)
    {
        const double ctr = 0.5 * (mn[d] + mx[d]);
        b.lo[d] = ctr - half;
        b.hi[d] = ctr + half;
    }
    b.periodic = 0;
    box_finish(b);
    *box = b;
}

__global__ void set_box_kernel(double x0, double x1, double y0, double y1, double z0, double z1, DevBox* box)
{
    if (threadIdx.x != 0) return;
    DevBox b;
    b.lo[0] = x0; b.hi[0] = x1; b.lo[1] = y0; b.hi[1] = y1; b.lo[2] = z0; b.hi[2] = z1;
    b.periodic = 1;
    box_finish(b);
    *box = b;
}

__global__ void keys_kernel(const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, const double* __restrict__ h, int n,
                            const DevBox* __restrict__ box, uint64_t* __restrict__ keys)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DevBox b = *box;
    uint64_t k = kDeadKey;
    if (h[i] > 0.0)
        k = hilbert_key(quantise(x[i], b.lo[0], b.scale[0]), quantise(y[i], b.lo[1], b.scale[1]),
                        quantise(z[i], b.lo[2], b.scale[2]));
    keys[i] = k;
}

// nAlive = first dead key (keys sorted).
__global__ void alive_kernel(const uint64_t* __restrict__ keys, int n, DevScalars* ds)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool dead = keys[i] == kDeadKey;
    const bool prevAlive = (i == 0) ? true : keys[i - 1] != kDeadKey;
    if (dead && prevAlive) ds->nAlive = int(i);
    if (!dead && i == n - 1) ds->nAlive = n;
}

// What a solve starts from zero, set by the gather (one pass over the particles instead
// of a memset per array): rho, gradh, the convergence flags and the Newton rows' h, the
// scalars' pair counters and hmax seen, and the index-row switch.
struct SolveReset
{
    double* rho;
    double* gradh;
    int* converged;
    double* rowH;
    DevScalars* ds;
    int rowsJOn;
};

__global__ void gather_particles_kernel(const int* __restrict__ order, int n,
                                        const double* __restrict__ ux, const double* __restrict__ uy,
                                        const double* __restrict__ uz, const double* __restrict__ uh,
                                        double4* __restrict__ xyzh, const double* __restrict__ uvx,
                                        const double* __restrict__ uvy, const double* __restrict__ uvz,
                                        const double* __restrict__ uax, const double* __restrict__ uay,
                                        const double* __restrict__ uaz, double4* __restrict__ vel4,
                                        double4* __restrict__ acc4, int alsoVA, SolveReset r)
{
    const long k = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k == 0)
    {
        for (int p = 0; p < 4; ++p) r.ds->pairs[p] = 0;
        r.ds->hmaxSeen = 0;
        r.ds->rowsJOn = r.rowsJOn;
    }
    if (k >= n) return;
    const int i = order[k];
    xyzh[k] = make_double4(ux[i], uy[i], uz[i], uh[i]);
    if (alsoVA)
    {
        vel4[k] = make_double4(uvx[i], uvy[i], uvz[i], 0.0);
        acc4[k] = make_double4(uax[i], uay[i], uaz[i], 0.0);
    }
    r.rho[k] = 0.0;
    r.gradh[k] = 0.0;
    r.converged[k] = 0;
    r.rowH[k] = 0.0;
}

// ------------------------------------------------------------------ leaf tree
__device__ __forceinline__ uint32_t lower_bound_u64(const uint64_t* a, uint32_t n, uint64_t v)
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

__global__ void leaf_count_kernel(const uint64_t* __restrict__ tree, int nL, const uint64_t* __restrict__ keys,
                                  const DevScalars* __restrict__ ds, uint32_t* __restrict__ counts,
                                  uint32_t* __restrict__ ops)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nL) return;
    const uint32_t na = uint32_t(ds->nAlive);
    const uint64_t a = tree[i], b = tree[i + 1];
    const uint32_t c = lower_bound_u64(keys, na, b) - lower_bound_u64(keys, na, a);
    counts[i] = c;
    const int L = level_of_range(b - a);
    ops[i] = (c > kBucket && L < kMaxLevel) ? 8u : 1u;
}

__global__ void leaf_split_kernel(const uint64_t* __restrict__ tree, int nL, const uint32_t* __restrict__ ops,
                                  const uint32_t* __restrict__ pos, uint64_t* __restrict__ out)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i > nL) return;
    if (i == nL) { out[pos[nL]] = kKeyEnd; return; }
    const uint64_t a = tree[i];
    const uint32_t p = pos[i];
    if (ops[i] == 8u)
    {
        const uint64_t child = (tree[i + 1] - a) >> 3;
        for (int o = 0; o < 8; ++o) out[p + o] = a + uint64_t(o) * child;
    }
    else out[p] = a;
}

// Where the leaf tree's refinement starts.  From the root, every node holding more than
// kBucket live particles splits into its eight children each round, so a node above the
// coarsest level at which some node holds kBucket or fewer is always split: the rounds
// that lead there produce the complete grid of that level whatever the particles.
// leaf_bounds_kernel finds where each of the 32768 level-5 cells starts in the sorted
// live keys (one binary search a thread); leaf_start_kernel takes each level's smallest
// count from those bounds and writes the complete grid of level L0 = 1 + the deepest
// level (at most 5) whose every node holds more than kBucket (0 when the root itself
// holds no more): 8^L0 leaves, their bounds in tree, the count in ds->leafStart.  When no
// node of that grid holds more than kBucket either (L0 at most 5, where its counts are
// known), the grid is the tree: its counts are written and ds->leafDone set.  Otherwise
// the rounds that follow from it give the tree the rounds from the root would.
constexpr int kStartLevels = 5;
constexpr int kStartCells = 1 << (3 * kStartLevels);

__global__ void leaf_bounds_kernel(const uint64_t* __restrict__ keys, DevScalars* __restrict__ ds,
                                   uint32_t* __restrict__ bounds)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > kStartCells) return;
    const uint32_t na = uint32_t(ds->nAlive);
    bounds[c] = c == kStartCells ? na
                                 : lower_bound_u64(keys, na, uint64_t(c) << (3 * (kMaxLevel - kStartLevels)));
}

__global__ void __launch_bounds__(1024)
leaf_start_kernel(const uint32_t* __restrict__ bounds, DevScalars* __restrict__ ds, uint64_t* __restrict__ tree,
                  uint32_t* __restrict__ counts)
{
    __shared__ uint32_t lmin[kStartLevels + 1], lmax[kStartLevels + 1];
    __shared__ int sL0;
    const uint32_t na = uint32_t(ds->nAlive);
    const int t = threadIdx.x;
    if (t <= kStartLevels)
    {
        lmin[t] = t == 0 ? na : 0xffffffffu;
        lmax[t] = t == 0 ? na : 0u;
    }
    __syncthreads();
    for (int l = 1; l <= kStartLevels; ++l)
    {
        const int cells = 1 << (3 * l), span = kStartCells / cells;
        for (int c = t; c < cells; c += blockDim.x)
        {
            const uint32_t k = bounds[(c + 1) * span] - bounds[c * span];
            atomicMin(&lmin[l], k);
            atomicMax(&lmax[l], k);
        }
    }
    __syncthreads();
    if (t == 0)
    {
        int L0 = 0;
        if (na > kBucket)
        {
            L0 = 1;
            for (int l = 1; l <= kStartLevels && lmin[l] > kBucket; ++l) L0 = l + 1;
        }
        sL0 = L0;
        ds->leafStart = 1 << (3 * L0);
        ds->leafDone = (L0 <= kStartLevels && lmax[L0] <= kBucket) ? 1 : 0;
    }
    __syncthreads();
    const int L0 = sL0, cells = 1 << (3 * L0);
    const bool done = L0 <= kStartLevels && lmax[L0] <= kBucket;
    const int span = L0 <= kStartLevels ? kStartCells / cells : 0;
    for (int c = t; c < cells; c += blockDim.x)
    {
        tree[c] = uint64_t(c) << (3 * (kMaxLevel - L0));
        if (done) counts[c] = bounds[(c + 1) * span] - bounds[c * span];
    }
    if (t == 0) tree[cells] = kKeyEnd;
}

// ------------------------------------------------------------------ linked octree
__device__ __forceinline__ int first_aligned_level(uint64_t k)
{
    if (k == 0) return 0;
    const int tz = __ffsll((long long)k) - 1;
    const int L0 = kMaxLevel - tz / 3;
    return L0 < 0 ? 0 : L0;
}

__global__ void node_count_kernel(const uint64_t* __restrict__ tree, int nL, uint32_t* __restrict__ cnt)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nL) return;
    const uint64_t k = tree[i];
    const int L = level_of_range(tree[i + 1] - k);
    const int L0 = first_aligned_level(k);
    cnt[i] = uint32_t((L > L0 ? L - L0 : 0) + 1);
}

// Pre-order emission: each leaf writes the internal nodes that start at its key
// (shallowest first) and then itself.  skip = size of the node's subtree in pre-order.
__global__ void node_emit_kernel(const uint64_t* __restrict__ tree, int nL, const uint32_t* __restrict__ start,
                                 int numNodes, uint64_t* __restrict__ prePrefix, int* __restrict__ preLeaf,
                                 int* __restrict__ preSkip)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nL) return;
    const uint64_t k = tree[i];
    const int L = level_of_range(tree[i + 1] - k);
    const int L0 = first_aligned_level(k);
    uint32_t pos = start[i];
    for (int a = (L0 < L ? L0 : L); a <= L; ++a, ++pos)
    {
        prePrefix[pos] = encode_prefix(k, a);
        preLeaf[pos] = (a == L) ? int(i) : -1;
        const uint64_t end = k + node_range(a);
        const uint32_t endLeaf = lower_bound_u64(tree, uint32_t(nL + 1), end);
        const uint32_t next = (endLeaf < uint32_t(nL)) ? start[endLeaf] : uint32_t(numNodes);
        preSkip[pos] = int(next - pos);
    }
}

__global__ void bfs_link_kernel(const uint64_t* __restrict__ bfsPrefix, const int* __restrict__ bfsToPre,
                                int numNodes, const int* __restrict__ preLeaf, int* __restrict__ preToBfs,
                                int* __restrict__ childOffsets, int* __restrict__ internalToLeaf,
                                int* __restrict__ leafToInternal, int* __restrict__ levelRange,
                                const DevBox* __restrict__ box, double* __restrict__ centers,
                                double* __restrict__ sizes, double4* __restrict__ preCenter,
                                double4* __restrict__ preHalf)
{
    const long b = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (b >= numNodes) return;
    const uint64_t p = bfsPrefix[b];
    const int pre = bfsToPre[b];
    preToBfs[pre] = int(b);
    const int leaf = preLeaf[pre];
    const int L = prefix_level(p);
    if (leaf >= 0)
    {
        childOffsets[b] = 0;
        internalToLeaf[b] = leaf;
        leafToInternal[leaf] = int(b);
    }
    else
    {
        childOffsets[b] = int(lower_bound_u64(bfsPrefix, uint32_t(numNodes), p << 3));
        internalToLeaf[b] = -1;
    }
    const int Lprev = (b == 0) ? -1 : prefix_level(bfsPrefix[b - 1]);
    for (int l = Lprev + 1; l <= L; ++l) levelRange[l] = int(b);
    if (b == numNodes - 1)
        for (int l = L + 1; l <= kMaxLevel + 1; ++l) levelRange[l] = numNodes;

    // Node geometry (include/tree.cuh:110-125): centre and half-size of the node's cube.
    uint32_t ic[3];
    hilbert_cell(prefix_start(p), ic[0], ic[1], ic[2]);
    const uint32_t side = 1u << (kMaxLevel - L);
    const double sd = double(side);
    const DevBox bx = *box;
    double c[3], s[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        const double corner = double(ic[d] & ~(side - 1u));
        c[d] = bx.lo[d] + (corner + 0.5 * sd) * bx.unit[d];
        s[d] = 0.5 * sd * bx.unit[d];
        centers[3 * b + d] = c[d];
        sizes[3 * b + d] = s[d];
    }
    preCenter[pre] = make_double4(c[0], c[1], c[2], 0.0);
    preHalf[pre] = make_double4(s[0], s[1], s[2], 0.0);
}

__global__ void particle_leaf_kernel(const uint32_t* __restrict__ layout, int nL, int nAliveMax,
                                     const DevScalars* __restrict__ ds, int* __restrict__ particleLeaf)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nAliveMax || i >= ds->nAlive) return;
    // last leaf whose start <= i, skipping empty leaves: upper_bound(layout, i) - 1
    uint32_t lo = 0, hi = uint32_t(nL + 1);
    while (lo < hi)
    {
        const uint32_t mid = (lo + hi) >> 1;
        if (layout[mid] <= uint32_t(i)) lo = mid + 1;
        else hi = mid;
    }
    particleLeaf[i] = int(lo) - 1;
}

__global__ void iota_kernel(int* __restrict__ a, int n)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) a[i] = int(i);
}

// ------------------------------------------------------------------ hmax
// include/tree.cuh:177-191: largest finite h of each listed leaf.
__global__ void hmax_leaf_kernel(const double4* __restrict__ xyzh, const uint32_t* __restrict__ layout,
                                 const int* __restrict__ leaves, int nActive, double* __restrict__ hmax,
                                 const int* __restrict__ countPtr, unsigned long long* __restrict__ seen)
{
    const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool on = t < (countPtr != nullptr ? *countPtr : nActive);
    double hm = 0.0;
    if (on)
    {
        const int l = leaves[t];
        for (uint32_t j = layout[l]; j < layout[l + 1]; ++j)
        {
            const double hj = xyzh[j].w;
            if (isfinite(hj)) hm = fmax(hm, hj);
        }
        hmax[l] = hm;
    }
    // the largest h of the solve so far, one atomic per warp (non-negative doubles order
    // as their bit patterns)
    if (seen != nullptr)
    {
        unsigned long long b = (unsigned long long)__double_as_longlong(hm);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
            const unsigned long long v = __shfl_xor_sync(0xffffffffu, b, o);
            b = v > b ? v : b;
        }
        if ((threadIdx.x & 31) == 0 && b != 0) atomicMax(seen, b);
    }
}

// include/tree.cuh:196-217, one level, deepest first.
__global__ void hmax_level_kernel(int first, int last, const int* __restrict__ childOffsets,
                                  const int* __restrict__ internalToLeaf, const double* __restrict__ hmaxLeaf,
                                  double* __restrict__ hmaxNode, const int* __restrict__ bfsToPre,
                                  double* __restrict__ hmaxPre)
{
    const int i = first + int(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= last) return;
    const int c = childOffsets[i];
    double m;
    if (c == 0)
    {
        const double hm = hmaxLeaf[internalToLeaf[i]];
        m = (isfinite(hm) && hm > 0.0) ? hm : 0.0;
    }
    else
    {
        m = 0.0;
        for (int o = 0; o < 8; ++o) m = fmax(m, hmaxNode[c + o]);
    }
    hmaxNode[i] = m;
    hmaxPre[bfsToPre[i]] = m;
}

constexpr double kListLoose = 1.05;   // a kept list may be this much wider than a new one

// ------------------------------------------------------------------ j-leaf list walk
// One warp per i-leaf.  The tree is scanned in pre-order 32 nodes at a time: every lane
// tests one node; the nodes before the first rejected one are all reached (an accepted
// node is followed by its successor in pre-order), so their leaves are emitted in order,
// and the scan resumes after the rejected node's subtree.  Accepted leaves therefore come
// out in ascending order, nothing is stacked, and nothing can be dropped.
// Gather test: a node is taken when its cell overlaps the i-leaf's cell widened by the
// search radius on every axis (include/tree.cuh's test, the lists callers read), or, with
// rounded set (the Newton loop's own lists), when its cell lies within the search radius
// of the i-leaf's cell -- the Euclidean gap, so the cube's corners are left out.  Every
// pair within the radius still has its j-leaf in the list, and a leaf with a large h
// near the edge of a concentrated set no longer takes in the dense centre its cube reaches.
template<bool Symmetric, bool Periodic, bool Fill>
__global__ void __launch_bounds__(kBlk, 5)
list_walk_kernel(int nL, int numNodes, const int* __restrict__ leafToInternal,
                 const double* __restrict__ centers, const double* __restrict__ sizes,
                 const double* __restrict__ hmaxLeaf, const double4* __restrict__ preCenter,
                 const double4* __restrict__ preHalf, const int* __restrict__ preSkip,
                 const int* __restrict__ preLeaf, const double* __restrict__ hmaxPre,
                 const DevBox* __restrict__ box, uint32_t* __restrict__ jcount,
                 const uint32_t* __restrict__ jOffset, int* __restrict__ jlist, int* err,
                 const uint32_t* __restrict__ layout, uint32_t* __restrict__ jstream, double margin,
                 double* __restrict__ listH, const uint32_t* __restrict__ jOffsetPrev,
                 const int* __restrict__ jlistPrev, int* __restrict__ walked, int* __restrict__ scratch,
                 int rounded, uint32_t streamCap, uint32_t listCap, const int* __restrict__ dims)
{
    const int lane = threadIdx.x & 31;
    const long leaf = (long(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (dims != nullptr)
    {
        // the leaf and node counts on the device (a captured graph); nL bounded them
        nL = dims[0];
        numNodes = dims[1];
    }
    if (leaf >= nL) return;
    // A fill writes only inside [jOffset[leaf], jOffset[leaf + 1]); a list storage of
    // listCap entries that the lists outgrew (a build whose total the host did not read
    // first) is reported, and nothing is written past it.
    if (Fill && jOffset[leaf + 1] > listCap)
    {
        if (lane == 0) atomicOr(err, int(kErrListFull));
        return;
    }
    // The count pass keeps the first kWalkScratch entries of every list it walks in
    // scratch; the fill pass copies a list that fitted instead of walking it again.
    if (Fill && scratch != nullptr && (walked == nullptr || walked[leaf] != 0))
    {
        const uint32_t dst = jOffset[leaf], cnt = jOffset[leaf + 1] - dst;
        if (cnt <= uint32_t(kWalkScratch))
        {
            const int* src = scratch + leaf * kWalkScratch;
            for (uint32_t k = lane; k < cnt; k += 32) jlist[dst + k] = src[k];
            return;
        }
    }
    double hmax = hmaxLeaf[leaf];
    if (!isfinite(hmax) || hmax <= 0.0) hmax = 0.0;
    // Incremental rebuild (walked set): a leaf whose hmax is still inside the radius its
    // previous list was walked at, and not so far inside that the list is looser than a
    // new one by more than kListLoose, keeps that list -- a superset, in the same
    // pre-order, of what this hmax needs -- and the fill pass copies it; the others walk.
    if (walked != nullptr)
    {
        if (!Fill && hmax <= listH[leaf] && listH[leaf] <= hmax * margin * kListLoose)
        {
            if (lane == 0)
            {
                jcount[leaf] = jOffsetPrev[leaf + 1] - jOffsetPrev[leaf];
                walked[leaf] = 0;
            }
            return;
        }
        if (Fill && walked[leaf] == 0)
        {
            const uint32_t dst = jOffset[leaf], cnt = jOffset[leaf + 1] - dst, src = jOffsetPrev[leaf];
            for (uint32_t k = lane; k < cnt; k += 32) jlist[dst + k] = jlistPrev[src + k];
            return;
        }
    }
    const int iNode = leafToInternal[leaf];
    const double icx = centers[3 * iNode], icy = centers[3 * iNode + 1], icz = centers[3 * iNode + 2];
    const double isx = sizes[3 * iNode], isy = sizes[3 * iNode + 1], isz = sizes[3 * iNode + 2];
    hmax *= margin;
    const double radHi = kRadKernel * hmax;
    // the rounded test's radius, with the slack of the group boxes (1e-9 of the radius,
    // 1e-13 of |centre|) above the rounding of the gaps.  It is used where the radius is
    // large against the cell (there the cube's corners hold most of its volume); for a
    // radius near the cell's size the cube test lists nearly the same leaves for less work.
    const double radR = radHi + 1e-9 * radHi + 1e-13 * (fabs(icx) + fabs(icy) + fabs(icz));
    const bool round = rounded && radHi > 4.0 * fmax(isx, fmax(isy, isz));
    // gather: the i-box inflated by radHi; symmetric: the raw i-box
    const double ax = Symmetric ? isx : isx + radHi;
    const double ay = Symmetric ? isy : isy + radHi;
    const double az = Symmetric ? isz : isz + radHi;
    double lx = 0, ly = 0, lz = 0;
    if (Periodic) { lx = box->len[0]; ly = box->len[1]; lz = box->len[2]; }

    uint32_t count = 0, base = 0, cap = 0, stream = 0;
    if (Fill) { base = jOffset[leaf]; cap = jOffset[leaf + 1] - base; }
    const uint32_t lt = (1u << lane) - 1u;

    int p = 0;
    while (p < numNodes)
    {
        const int idx = p + lane;
        const bool valid = idx < numNodes;
        bool accept = false;
        int skip = 1, pl = -1;
        if (valid)
        {
            const double4 c = preCenter[idx];
            const double4 s = preHalf[idx];
            double dd[3] = {fabs(icx - c.x), fabs(icy - c.y), fabs(icz - c.z)};
            if (Periodic)
            {
                dd[0] = fmin(dd[0], lx - dd[0]);
                dd[1] = fmin(dd[1], ly - dd[1]);
                dd[2] = fmin(dd[2], lz - dd[2]);
            }
            const double g0 = dd[0] - ax - s.x, g1 = dd[1] - ay - s.y, g2 = dd[2] - az - s.z;
            const double d0 = (g0 > 0.0) ? g0 : 0.0, d1 = (g1 > 0.0) ? g1 : 0.0, d2 = (g2 > 0.0) ? g2 : 0.0;
            const double n2 = d0 * d0 + d1 * d1 + d2 * d2;
            if (Symmetric)
            {
                const double rs = fmax(radHi, kRadKernel * hmaxPre[idx]);
                accept = n2 <= rs * rs;
            }
            else if (round)
            {
                const double e0 = fmax(dd[0] - isx - s.x, 0.0), e1 = fmax(dd[1] - isy - s.y, 0.0);
                const double e2 = fmax(dd[2] - isz - s.z, 0.0);
                accept = e0 * e0 + e1 * e1 + e2 * e2 <= radR * radR;
            }
            else accept = n2 <= 0.0;
            skip = preSkip[idx];
            pl = preLeaf[idx];
        }
        const uint32_t validMask = __ballot_sync(0xffffffffu, valid);
        const uint32_t rejMask = __ballot_sync(0xffffffffu, valid && !accept);
        // Walk the window: runs of reached nodes end at a rejection, after which the scan
        // jumps over that node's subtree; a jump that lands inside the window continues.
        int pos = 0;        // offset of the next reached node in this window
        int next = p + 32;  // where the following window starts
        for (;;)
        {
            const uint32_t fromPos = (pos >= 32) ? 0u : (0xffffffffu << pos);
            const uint32_t rej = rejMask & fromPos;
            const int r = rej ? (__ffs(rej) - 1) : 32;
            // lanes [pos, r) are reached and accepted
            const uint32_t runMask = validMask & fromPos & ((r >= 32) ? 0xffffffffu : ((1u << r) - 1u));
            const uint32_t emitMask = __ballot_sync(0xffffffffu, ((runMask >> lane) & 1u) && pl >= 0);
            if (Fill)
            {
                if ((emitMask >> lane) & 1u)
                {
                    const uint32_t slot = count + __popc(emitMask & lt);
                    if (slot < cap) jlist[base + slot] = pl;
                    else atomicOr(err, int(kErrListCap));
                }
            }
            else if ((emitMask >> lane) & 1u)
            {
                if (jstream != nullptr) stream += layout[pl + 1] - layout[pl];
                const uint32_t slot = count + __popc(emitMask & lt);
                if (scratch != nullptr && slot < uint32_t(kWalkScratch)) scratch[leaf * kWalkScratch + slot] = pl;
            }
            count += __popc(emitMask);
            if (r >= 32) { next = p + 32; break; }
            int rskip = __shfl_sync(0xffffffffu, skip, r);
            if (rskip < 1) rskip = 1;   // a subtree holds its root: the scan always advances
            const int target = p + r + rskip;
            if (target >= p + 32 || target >= numNodes) { next = target; break; }
            pos = target - p;
        }
        p = next;
        // A count walk with a stream cap stops once the list streams more than the cap:
        // such a leaf is cut into one-particle groups that scan the tree for their own
        // spheres (the cut gives one particle per group at any stream above the cut's
        // work figure, which is the cap), so the list itself is never read.  It is left
        // empty and its stream marked as unbounded.  The stream is summed over the lanes
        // only once the listed leaves could hold more than the cap (kBucket each, leaves
        // at the deepest level aside: missing one of those only walks a list in full).
        if (!Fill && streamCap != 0u && jstream != nullptr && uint64_t(count) * kBucket > streamCap &&
            __reduce_add_sync(0xffffffffu, stream) > streamCap)
        {
            if (lane == 0)
            {
                jcount[leaf] = 0;
                jstream[leaf] = 0xffffffffu;
                if (listH != nullptr) listH[leaf] = hmax;
                if (walked != nullptr) walked[leaf] = 1;
            }
            return;
        }
    }
    if (!Fill && jstream != nullptr)
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
            if (jstream != nullptr) jstream[leaf] = stream;
            if (listH != nullptr) listH[leaf] = hmax;
            if (walked != nullptr) walked[leaf] = 1;
        }
    }
}

} // namespace

// ====================================================================== host side
uint32_t scan_exclusive(State& s, const uint32_t* in, uint32_t* out, int n, bool readTotal)
{
    const int nb = std::max(1, iceil(n, kScanTile));
    if (nb > kScanTile) fatal("scan_exclusive: %d elements exceed the scan capacity", n);
    s.scanTmp.resize(size_t(nb) + 1, s.st);
    uint32_t* bsum = s.scanTmp.get();
    scan_reduce_kernel<<<nb, kScanThreads, 0, s.st>>>(in, n, bsum);
    COSMO_LAUNCHED();
    scan_blocks_kernel<<<1, kScanThreads, 0, s.st>>>(bsum, nb, out + n);
    COSMO_LAUNCHED();
    scan_apply_kernel<<<nb, kScanThreads, 0, s.st>>>(in, out, n, bsum);
    COSMO_LAUNCHED();
    if (!readTotal) return 0;
    COSMO_CUDA(cudaMemcpyAsync(s.hsmall, out + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s.st));
    COSMO_CUDA(cudaStreamSynchronize(s.st));
    return uint32_t(s.hsmall[0]);
}

void scan_reserve(State& s, int nCap)
{
    s.scanTmp.resize(size_t(std::max(1, iceil(nCap, kScanTile))) + 1, s.st);
}

void scan_exclusive_dev(State& s, const uint32_t* in, uint32_t* out, int nCap, const int* nPtr)
{
    const int nb = std::max(1, iceil(nCap, kScanTile));
    if (nb > kScanTile) fatal("scan_exclusive: %d elements exceed the scan capacity", nCap);
    s.scanTmp.resize(size_t(nb) + 1, s.st);
    uint32_t* bsum = s.scanTmp.get();
    scan_reduce_kernel<<<nb, kScanThreads, 0, s.st>>>(in, nCap, bsum, nPtr);
    COSMO_LAUNCHED();
    scan_blocks_kernel<<<1, kScanThreads, 0, s.st>>>(bsum, nb, nullptr, out, nPtr);
    COSMO_LAUNCHED();
    scan_apply_kernel<<<nb, kScanThreads, 0, s.st>>>(in, out, nCap, bsum, nPtr);
    COSMO_LAUNCHED();
}

__global__ void level_keys_kernel(const uint64_t* __restrict__ prefix, int n, uint64_t* __restrict__ lvl)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) lvl[i] = uint64_t(prefix_level(prefix[i]));
}

__global__ void gather_prefix_kernel(const uint64_t* __restrict__ prePrefix, const int* __restrict__ bfsToPre, int n,
                                     uint64_t* __restrict__ bfsPrefix)
{
    const long b = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (b < n) bfsPrefix[b] = prePrefix[bfsToPre[b]];
}

// bfsToPre / bfsPrefix: the pre-order nodes partitioned stably by level (one onesweep
// pass on the level, below 256), which is their order by prefix.
static void sort_nodes_by_level(State& s, int n)
{
    const int tiles = iceil(n, kSortTile);
    s.sortHist.resize(kSortPasses * 256, s.st);
    s.sortBase.resize(kSortPasses * 256, s.st);
    s.sortLookback.resize(size_t(kSortPasses) * tiles * 256, s.st);
    DevScalars* ds = s.dscal.get();
    COSMO_CUDA(cudaMemsetAsync(s.sortHist.get(), 0, kSortPasses * 256 * sizeof(uint32_t), s.st));
    COSMO_CUDA(cudaMemsetAsync(s.sortLookback.get(), 0, size_t(tiles) * 256 * sizeof(uint32_t), s.st));
    COSMO_CUDA(cudaMemsetAsync(&ds->sortTiles[0], 0, sizeof(unsigned int), s.st));
    level_keys_kernel<<<iceil(n, kBlk), kBlk, 0, s.st>>>(s.prePrefix.get(), n, s.nodeKeysTmp.get());
    COSMO_LAUNCHED();
    digit_hist_kernel<<<std::min(iceil(n, kBlk), 4 * s.numSMs), kBlk, 0, s.st>>>(s.nodeKeysTmp.get(), n,
                                                                                 s.sortHist.get());
    COSMO_LAUNCHED();
    digit_base_kernel<<<kSortPasses, 256, 0, s.st>>>(s.sortHist.get(), s.sortBase.get());
    COSMO_LAUNCHED();
    // keys out into bfsPrefix (overwritten by the gather below), pre-order indices into bfsToPre
    onesweep_kernel<<<tiles, kSortThreads, 0, s.st>>>(s.nodeKeysTmp.get(), nullptr, s.bfsPrefix.get(),
                                                     s.bfsToPre.get(), n, 0, s.sortBase.get(), s.sortLookback.get(),
                                                     &ds->sortTiles[0], &ds->err, wait_limit_ns());
    COSMO_LAUNCHED();
    gather_prefix_kernel<<<iceil(n, kBlk), kBlk, 0, s.st>>>(s.prePrefix.get(), s.bfsToPre.get(), n,
                                                            s.bfsPrefix.get());
    COSMO_LAUNCHED();
}

void radix_sort_u64(State& s, uint64_t* kA, uint64_t* kB, int* vA, int* vB, int n, bool iotaValues)
{
    if (n <= 0) return;
    const int tiles = iceil(n, kSortTile);
    s.sortHist.resize(kSortPasses * 256, s.st);
    s.sortBase.resize(kSortPasses * 256, s.st);
    s.sortLookback.resize(size_t(kSortPasses) * tiles * 256, s.st);
    DevScalars* ds = s.dscal.get();
    COSMO_CUDA(cudaMemsetAsync(s.sortHist.get(), 0, kSortPasses * 256 * sizeof(uint32_t), s.st));
    COSMO_CUDA(cudaMemsetAsync(s.sortLookback.get(), 0, size_t(kSortPasses) * tiles * 256 * sizeof(uint32_t), s.st));
    COSMO_CUDA(cudaMemsetAsync(&ds->sortTiles[0], 0, sizeof(ds->sortTiles), s.st));
    digit_hist_kernel<<<std::min(iceil(n, kBlk), 4 * s.numSMs), kBlk, 0, s.st>>>(kA, n, s.sortHist.get());
    COSMO_LAUNCHED();
    digit_base_kernel<<<kSortPasses, 256, 0, s.st>>>(s.sortHist.get(), s.sortBase.get());
    COSMO_LAUNCHED();
    uint64_t* ki = kA; uint64_t* ko = kB;
    int* vi = iotaValues ? nullptr : vA; int* vo = vB;
    for (int p = 0; p < kSortPasses; ++p)
    {
        onesweep_kernel<<<tiles, kSortThreads, 0, s.st>>>(
            ki, vi, ko, vo, n, 8 * p, s.sortBase.get() + 256 * p,
            s.sortLookback.get() + size_t(p) * tiles * 256, &ds->sortTiles[p], &ds->err, wait_limit_ns());
        COSMO_LAUNCHED();
        std::swap(ki, ko);
        vi = vo;
        vo = (vo == vB) ? vA : vB;
    }
    // eight passes: the result is back in kA / vA
}

// ---------------------------------------------------------------------------------------
// Hilbert keys and their stable sort with every buffer supplied by the caller (used by
// the allocation-free entry point in noalloc.cu).  Same kernels and launch sequence as
// build_tree's keys + radix_sort_u64; scratch is carved as laid out below.
// ---------------------------------------------------------------------------------------
namespace {
constexpr size_t kAlign = 256;
inline size_t align_up(size_t v) { return (v + kAlign - 1) & ~(kAlign - 1); }
constexpr int kRawBboxBlocks = 296;
}

size_t keysort_scratch_bytes(int n)
{
    const size_t tiles = size_t(std::max(1, iceil(n, kSortTile)));
    size_t b = 0;
    b += align_up(sizeof(DevBox));
    b += align_up(size_t(kRawBboxBlocks) * 6 * sizeof(double));
    b += align_up(kSortPasses * 256 * sizeof(uint32_t));       // histograms
    b += align_up(kSortPasses * 256 * sizeof(uint32_t));       // bin bases
    b += align_up(16 * sizeof(unsigned int) + sizeof(int));    // tile tickets + error word
    b += align_up(size_t(kSortPasses) * tiles * 256 * sizeof(uint32_t));
    b += align_up(size_t(n) * sizeof(uint64_t));               // key ping-pong partner
    b += align_up(size_t(n) * sizeof(int));                    // index ping-pong partner
    return b;
}

int keysort_raw(int n, const double* x, const double* y, const double* z, const double* h,
                const double* periodicBox, uint64_t* keysOut, int* orderOut, void* scratch, int numSMs,
                cudaStream_t st)
{
    const int tiles = std::max(1, iceil(n, kSortTile));
    char* p = static_cast<char*>(scratch);
    auto take = [&](size_t bytes) { char* q = p; p += align_up(bytes); return q; };
    DevBox* box = reinterpret_cast<DevBox*>(take(sizeof(DevBox)));
    double* part = reinterpret_cast<double*>(take(size_t(kRawBboxBlocks) * 6 * sizeof(double)));
    uint32_t* hist = reinterpret_cast<uint32_t*>(take(kSortPasses * 256 * sizeof(uint32_t)));
    uint32_t* base = reinterpret_cast<uint32_t*>(take(kSortPasses * 256 * sizeof(uint32_t)));
    unsigned int* tickets = reinterpret_cast<unsigned int*>(take(16 * sizeof(unsigned int) + sizeof(int)));
    int* err = reinterpret_cast<int*>(tickets + 16);
    uint32_t* lookback = reinterpret_cast<uint32_t*>(take(size_t(kSortPasses) * tiles * 256 * sizeof(uint32_t)));
    uint64_t* kB = reinterpret_cast<uint64_t*>(take(size_t(n) * sizeof(uint64_t)));
    int* vB = reinterpret_cast<int*>(take(size_t(n) * sizeof(int)));

    // The array keeps the previous call's contents: clear what must start at zero.
    if (cudaMemsetAsync(hist, 0, kSortPasses * 256 * sizeof(uint32_t), st) != cudaSuccess) return -2;
    if (cudaMemsetAsync(tickets, 0, 16 * sizeof(unsigned int) + sizeof(int), st) != cudaSuccess) return -2;
    if (cudaMemsetAsync(lookback, 0, size_t(kSortPasses) * tiles * 256 * sizeof(uint32_t), st) != cudaSuccess)
        return -2;
    if (periodicBox)
        set_box_kernel<<<1, 32, 0, st>>>(periodicBox[0], periodicBox[1], periodicBox[2], periodicBox[3],
                                         periodicBox[4], periodicBox[5], box);
    else
    {
        const int nb = std::min(std::min(iceil(n, kBlk), 2 * numSMs), kRawBboxBlocks);
        bbox_partial_kernel<<<nb, kBlk, 0, st>>>(x, y, z, n, part);
        bbox_final_kernel<<<1, 32, 0, st>>>(part, nb, box);
    }
    keys_kernel<<<iceil(n, kBlk), kBlk, 0, st>>>(x, y, z, h, n, box, keysOut);
    digit_hist_kernel<<<std::min(iceil(n, kBlk), 4 * numSMs), kBlk, 0, st>>>(keysOut, n, hist);
    digit_base_kernel<<<kSortPasses, 256, 0, st>>>(hist, base);
    uint64_t* ki = keysOut; uint64_t* ko = kB;
    int* vi = nullptr; int* vo = vB;
    for (int pass = 0; pass < kSortPasses; ++pass)
    {
        onesweep_kernel<<<tiles, kSortThreads, 0, st>>>(ki, vi, ko, vo, n, 8 * pass, base + 256 * pass,
                                                        lookback + size_t(pass) * tiles * 256, &tickets[pass], err,
                                                        wait_limit_ns());
        std::swap(ki, ko);
        vi = vo;
        vo = (vo == vB) ? orderOut : vB;
    }
    if (cudaGetLastError() != cudaSuccess) return -2;
    int e = 0;
    if (cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return -2;
    if (cudaStreamSynchronize(st) != cudaSuccess) return -2;
    return e ? -3 : 0;
}

void build_tree(State& s, const double* periodicBox, bool alsoSortVA, bool rowsJOn)
{
    const int n = s.ngas;
    DevScalars* ds = s.dscal.get();
    cudaEvent_t e0 = ev(s);

    // bounding box (src/tree.cu:47-72)
    if (periodicBox)
    {
        set_box_kernel<<<1, 32, 0, s.st>>>(periodicBox[0], periodicBox[1], periodicBox[2], periodicBox[3],
                                            periodicBox[4], periodicBox[5], s.box.get());
    }
    else if (s.keyExtentSet)
    {
        // the caller's extents (a rank of a decomposed set: the whole set's), through the
        // same box construction
        s.redTmp.resize(6, s.st);
        const double* e = s.keyExtent;
        set_extent_kernel<<<1, 32, 0, s.st>>>(s.redTmp.get(), e[0], e[1], e[2], e[3], e[4], e[5]);
        COSMO_LAUNCHED();
        bbox_final_kernel<<<1, 32, 0, s.st>>>(s.redTmp.get(), 1, s.box.get());
    }
    else
    {
        const int nb = std::min(iceil(n, kBlk), 2 * s.numSMs);
        s.redTmp.resize(size_t(nb) * 6, s.st);
        bbox_partial_kernel<<<nb, kBlk, 0, s.st>>>(s.ux.get(), s.uy.get(), s.uz.get(), n, s.redTmp.get());
        COSMO_LAUNCHED();
        bbox_final_kernel<<<1, 32, 0, s.st>>>(s.redTmp.get(), nb, s.box.get());
    }
    COSMO_LAUNCHED();
    cudaEvent_t e1 = ev(s);

    // keys and sort (src/tree.cu:82-108)
    keys_kernel<<<iceil(n, kBlk), kBlk, 0, s.st>>>(s.ux.get(), s.uy.get(), s.uz.get(), s.uh.get(), n,
                                                  s.box.get(), s.keysA.get());
    COSMO_LAUNCHED();
    radix_sort_u64(s, s.keysA.get(), s.keysB.get(), s.orderA.get(), s.orderB.get(), n, true);
    alive_kernel<<<iceil(n, kBlk), kBlk, 0, s.st>>>(s.keysA.get(), n, ds);
    COSMO_LAUNCHED();
    s.nblH.resize(std::max(n, 1), s.st);
    gather_particles_kernel<<<iceil(std::max(n, 1), kBlk), kBlk, 0, s.st>>>(
        s.orderA.get(), n, s.ux.get(), s.uy.get(), s.uz.get(), s.uh.get(), s.xyzh.get(), s.uvx.get(),
        s.uvy.get(), s.uvz.get(), s.uax.get(), s.uay.get(), s.uaz.get(), s.vel4.get(), s.acc4.get(),
        alsoSortVA ? 1 : 0,
        SolveReset{s.rho.get(), s.gradh.get(), s.converged.get(), s.nblH.get(), ds, rowsJOn ? 1 : 0});
    COSMO_LAUNCHED();
    cudaEvent_t e2 = ev(s);

    // cornerstone leaf tree (src/tree.cu:126-136): the refinement from the root, started at
    // the complete grid of the level above which every node splits
    s.csTree.resize((size_t(1) << (3 * kStartLevels + 3)) + 1, s.st);
    s.startBounds.resize(kStartCells + 1, s.st);
    s.counts.resize(kStartCells, s.st);
    leaf_bounds_kernel<<<iceil(kStartCells + 1, 256), 256, 0, s.st>>>(s.keysA.get(), ds, s.startBounds.get());
    COSMO_LAUNCHED();
    leaf_start_kernel<<<1, 1024, 0, s.st>>>(s.startBounds.get(), ds, s.csTree.get(), s.counts.get());
    COSMO_LAUNCHED();
    read_scalars(s);
    s.nAlive = s.hscal->nAlive;   // counted by alive_kernel before the gather
    int nL = s.hscal->leafStart;
    const bool startIsTree = s.hscal->leafDone != 0;
    for (int round = 0; round < 64 && !startIsTree; ++round)
    {
        s.counts.resize(nL, s.st);
        s.ops.resize(nL, s.st);
        s.opsScan.resize(size_t(nL) + 1, s.st);
        leaf_count_kernel<<<iceil(nL, kBlk), kBlk, 0, s.st>>>(s.csTree.get(), nL, s.keysA.get(), ds,
                                                             s.counts.get(), s.ops.get());
        COSMO_LAUNCHED();
        const int total = int(scan_exclusive(s, s.ops.get(), s.opsScan.get(), nL, true));
        if (total == nL) break;
        s.csTree2.resize(size_t(total) + 1, s.st);
        leaf_split_kernel<<<iceil(nL + 1, kBlk), kBlk, 0, s.st>>>(s.csTree.get(), nL, s.ops.get(),
                                                                  s.opsScan.get(), s.csTree2.get());
        COSMO_LAUNCHED();
        std::swap(s.csTree, s.csTree2);
        nL = total;
    }
    s.nLeaves = nL;
    s.layout.resize(size_t(nL) + 1, s.st);
    scan_exclusive(s, s.counts.get(), s.layout.get(), nL, false);

    // linked octree: pre-order emission, then BFS order by sorting the prefixes
    s.nodeCount.resize(nL, s.st);
    s.leafPreStart.resize(size_t(nL) + 1, s.st);
    node_count_kernel<<<iceil(nL, kBlk), kBlk, 0, s.st>>>(s.csTree.get(), nL, s.nodeCount.get());
    COSMO_LAUNCHED();
    // every internal node of the refinement has eight children, so the octree of nL leaves
    // has (nL - 1) / 7 internal nodes: the node count needs no read of the scan's total
    scan_exclusive(s, s.nodeCount.get(), s.leafPreStart.get(), nL, false);
    const int numNodes = nL + (nL - 1) / 7;
    s.numNodes = numNodes;
    for (auto* b : {&s.prePrefix, &s.bfsPrefix}) b->resize(numNodes, s.st);
    for (auto* b : {&s.preLeaf, &s.preSkip, &s.bfsToPre, &s.preToBfs, &s.childOffsets, &s.internalToLeaf})
        b->resize(numNodes, s.st);
    s.centers.resize(size_t(3) * numNodes, s.st);
    s.sizes.resize(size_t(3) * numNodes, s.st);
    s.preCenter.resize(numNodes, s.st);
    s.preHalf.resize(numNodes, s.st);
    s.levelRange.resize(kMaxLevel + 2, s.st);
    s.leafToInternal.resize(nL, s.st);
    node_emit_kernel<<<iceil(nL, kBlk), kBlk, 0, s.st>>>(s.csTree.get(), nL, s.leafPreStart.get(), numNodes,
                                                         s.prePrefix.get(), s.preLeaf.get(), s.preSkip.get());
    COSMO_LAUNCHED();
    // BFS order = the nodes sorted by prefix, i.e. by (level, key).  Pre-order already has
    // every level's nodes in ascending key, so the sort is a stable partition of the
    // pre-order sequence by level: one counting pass on the level.
    s.nodeKeysTmp.resize(numNodes, s.st);
    sort_nodes_by_level(s, numNodes);
    cudaEvent_t e3 = ev(s);

    bfs_link_kernel<<<iceil(numNodes, kBlk), kBlk, 0, s.st>>>(
        s.bfsPrefix.get(), s.bfsToPre.get(), numNodes, s.preLeaf.get(), s.preToBfs.get(),
        s.childOffsets.get(), s.internalToLeaf.get(), s.leafToInternal.get(), s.levelRange.get(), s.box.get(),
        s.centers.get(), s.sizes.get(), s.preCenter.get(), s.preHalf.get());
    COSMO_LAUNCHED();
    particle_leaf_kernel<<<iceil(n, kBlk), kBlk, 0, s.st>>>(s.layout.get(), nL, n, ds, s.particleLeaf.get());
    COSMO_LAUNCHED();
    s.hmaxLeaf.resize(nL, s.st);
    s.hmaxNode.resize(numNodes, s.st);
    s.hmaxPre.resize(numNodes, s.st);
    s.jcount.resize(nL, s.st);
    s.jstream.resize(nL, s.st);
    s.listH.resize(nL, s.st);
    s.jOffset.resize(size_t(nL) + 1, s.st);
    s.allLeaves.resize(nL, s.st);
    iota_kernel<<<iceil(nL, kBlk), kBlk, 0, s.st>>>(s.allLeaves.get(), nL);
    COSMO_LAUNCHED();
    cudaEvent_t e4 = ev(s);
    // the stage times are taken once the stream has been read again (tree_timings)
    const cudaEvent_t marks[5] = {e0, e1, e2, e3, e4};
    std::copy(marks, marks + 5, s.treeEv);
}

void tree_timings(State& s)
{
    if (!s.treeEv[4]) return;
    COSMO_CUDA(cudaEventSynchronize(s.treeEv[4]));
    s.t.bbox += elapsed_s(s.treeEv[0], s.treeEv[1]);
    s.t.keysSort += elapsed_s(s.treeEv[1], s.treeEv[2]);
    s.t.tree += elapsed_s(s.treeEv[2], s.treeEv[3]);
    s.t.nodes += elapsed_s(s.treeEv[3], s.treeEv[4]);
    s.treeEv[4] = nullptr;
}

void hmax_leaves(State& s, const int* leaves, int nActive, const int* countPtr)
{
    if (nActive <= 0) return;
    hmax_leaf_kernel<<<iceil(nActive, kBlk), kBlk, 0, s.st>>>(s.xyzh.get(), s.layout.get(), leaves, nActive,
                                                             s.hmaxLeaf.get(), countPtr, &s.dscal.get()->hmaxSeen);
    COSMO_LAUNCHED();
}

void hmax_upsweep(State& s)
{
    int lr[kMaxLevel + 2];
    COSMO_CUDA(cudaMemcpyAsync(s.hsmall, s.levelRange.get(), sizeof(lr), cudaMemcpyDeviceToHost, s.st));
    COSMO_CUDA(cudaStreamSynchronize(s.st));
    std::copy(s.hsmall, s.hsmall + kMaxLevel + 2, lr);
    for (int L = kMaxLevel; L >= 0; --L)
    {
        const int a = lr[L], b = lr[L + 1];
        if (b <= a) continue;
        hmax_level_kernel<<<iceil(b - a, kBlk), kBlk, 0, s.st>>>(a, b, s.childOffsets.get(), s.internalToLeaf.get(),
                                                                 s.hmaxLeaf.get(), s.hmaxNode.get(),
                                                                 s.bfsToPre.get(), s.hmaxPre.get());
        COSMO_LAUNCHED();
    }
}

template<bool Sym, bool Per>
static void walk(State& s, bool fill, double margin, bool incremental, bool rounded, uint32_t streamCap,
                 const int* dims = nullptr, int leafCap = 0)
{
    const int nL = dims ? leafCap : s.nLeaves;
    const int blocks = iceil(long(nL) * 32, kBlk);
    auto args = [&](auto kern) {
        kern<<<blocks, kBlk, 0, s.st>>>(nL, s.numNodes, s.leafToInternal.get(), s.centers.get(), s.sizes.get(),
                                        s.hmaxLeaf.get(), s.preCenter.get(), s.preHalf.get(), s.preSkip.get(),
                                        s.preLeaf.get(), s.hmaxPre.get(), s.box.get(), s.jcount.get(),
                                        s.jOffset.get(), s.jlist.get(), &s.dscal.get()->err, s.layout.get(),
                                        !fill ? s.jstream.get() : nullptr, margin,
                                        (!fill && !Sym) ? s.listH.get() : nullptr,
                                        incremental ? s.jOffsetPrev.get() : nullptr,
                                        incremental ? s.jlistPrev.get() : nullptr,
                                        incremental ? s.walked.get() : nullptr, s.walkScratch.get(),
                                        rounded ? 1 : 0, streamCap,
                                        uint32_t(std::min<size_t>(s.listStore ? s.listStore : s.jlist.cap, 0xffffffffu)),
                                        dims);
    };
    if (fill) args(list_walk_kernel<Sym, Per, true>);
    else args(list_walk_kernel<Sym, Per, false>);
    COSMO_LAUNCHED();
}

// Copy the lists' entries [0, jOffset[*nL]) (counts on the device) into dst.
__global__ void copy_list_kernel(const int* __restrict__ src, int* __restrict__ dst, const uint32_t* __restrict__ jOffset,
                                 const int* __restrict__ nL)
{
    const uint32_t n = jOffset[*nL];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i];
}

// The Newton loop's incremental rebuild of the gather lists with no host read: the
// current lists are kept aside (their total read on the device), the outgrown leaves
// walk, and the fill writes into the storage already held (jlist.cap entries); a build
// that would not fit raises kErrListFull and writes nothing past it.  Every size is fixed
// when it is issued, so the sequence can be captured into a graph.
void build_lists_device(State& s, double margin, bool rounded, uint32_t streamCap, const int* dims, int leafCap)
{
    COSMO_CUDA(cudaMemcpyAsync(s.jOffsetPrev.get(), s.jOffset.get(), (size_t(leafCap) + 1) * sizeof(uint32_t),
                               cudaMemcpyDeviceToDevice, s.st));
    copy_list_kernel<<<4 * s.numSMs, 256, 0, s.st>>>(s.jlist.get(), s.jlistPrev.get(), s.jOffset.get(), dims);
    COSMO_LAUNCHED();
    if (s.periodic) walk<false, true>(s, false, margin, true, rounded, streamCap, dims, leafCap);
    else walk<false, false>(s, false, margin, true, rounded, streamCap, dims, leafCap);
    scan_exclusive_dev(s, s.jcount.get(), s.jOffset.get(), leafCap, dims);
    if (s.periodic) walk<false, true>(s, true, margin, true, rounded, streamCap, dims, leafCap);
    else walk<false, false>(s, true, margin, true, rounded, streamCap, dims, leafCap);
}

// include/tree.cuh:360-389: count, scan, size, fill -- for ALL leaves.  incremental
// (gather lists only, over the gather lists of the same tree at the same margin): the
// current lists are kept aside first, and only the leaves whose hmax outgrew them walk.
void build_lists(State& s, bool symmetric, double margin, bool incremental, bool rounded, uint32_t streamCap)
{
    rounded = rounded && !symmetric;
    if (symmetric || !rounded) streamCap = 0;   // the lists a caller reads are always whole
    const int nL = s.nLeaves;
    incremental = incremental && !symmetric && !s.listsSym && nL > 0;
    if (incremental)
    {
        s.jOffsetPrev.resize(size_t(nL) + 1, s.st);
        s.jlistPrev.resize(std::max<uint32_t>(s.listTotal, 1u), s.st);
        s.walked.resize(nL, s.st);
        COSMO_CUDA(cudaMemcpyAsync(s.jOffsetPrev.get(), s.jOffset.get(), (size_t(nL) + 1) * sizeof(uint32_t),
                                   cudaMemcpyDeviceToDevice, s.st));
        if (s.listTotal > 0)
            COSMO_CUDA(cudaMemcpyAsync(s.jlistPrev.get(), s.jlist.get(), size_t(s.listTotal) * sizeof(int),
                                       cudaMemcpyDeviceToDevice, s.st));
    }
    s.walkScratch.resize(size_t(nL) * kWalkScratch, s.st);
    auto run = [&](bool fill) {
        if (symmetric)
        {
            if (s.periodic) walk<true, true>(s, fill, margin, false, false, 0u);
            else walk<true, false>(s, fill, margin, false, false, 0u);
        }
        else
        {
            if (s.periodic) walk<false, true>(s, fill, margin, incremental, rounded, streamCap);
            else walk<false, false>(s, fill, margin, incremental, rounded, streamCap);
        }
    };
    run(false);
    const uint32_t total = scan_exclusive(s, s.jcount.get(), s.jOffset.get(), nL, true);
    s.jlist.resize(std::max<uint32_t>(total, 1u), s.st);
    run(true);
    s.listTotal = total;
    s.listsSym = symmetric;
}

} // namespace cosmo
