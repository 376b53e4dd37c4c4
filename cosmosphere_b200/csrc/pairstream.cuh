/*
 * pairstream.cuh -- the j-stream shared by the density, gradient and force kernels.
 *
 * A warp owns one group of up to 32 i-particles of one leaf (one per lane).  It walks
 * the leaf's j-leaf list in ascending order, loading 32 consecutive j particles per
 * batch with coalesced 128-bit loads.  Each j is tested ONCE, by the lane that loaded
 * it, against a conservative box around the whole group (the "group filter"); the
 * survivors are compacted with a ballot, in order, into a per-warp shared-memory ring,
 * and every lane then evaluates them one by one (broadcast reads).  A j rejected by the
 * filter cannot be accepted by any lane's exact test, so the accepted pairs -- and the
 * order in which each lane sums them -- are exactly those of walking the whole list.
 */
#pragma once

#include "common.cuh"
#include "tma.cuh"

namespace cosmo {

constexpr int kRing = 64;     // double4 entries per warp ring (2 KB)

// Conservative box of a group: centre c, half extents e (inflated by the caller's
// support and a rounding margin), and the periodic lengths.
struct GroupBox
{
    double cx, cy, cz, ex, ey, ez;
};

__device__ __forceinline__ double warp_min(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Box of [x - r, x + r] over the lanes that own a particle, plus an absolute margin far
// above the rounding of any coordinate involved (1e-9 of the support, 1e-13 of |c|).
__device__ __forceinline__ GroupBox group_box(bool mine, double x, double y, double z, double r, double rmax)
{
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    const double lx = warp_min(mine ? x - r : inf), hx = warp_max(mine ? x + r : -inf);
    const double ly = warp_min(mine ? y - r : inf), hy = warp_max(mine ? y + r : -inf);
    const double lz = warp_min(mine ? z - r : inf), hz = warp_max(mine ? z + r : -inf);
    GroupBox b;
    b.cx = 0.5 * (lx + hx); b.cy = 0.5 * (ly + hy); b.cz = 0.5 * (lz + hz);
    const double mx = 1e-9 * rmax + 1e-13 * (fabs(b.cx) + fabs(b.cy) + fabs(b.cz) + 1e-300);
    b.ex = 0.5 * (hx - lx) + mx; b.ey = 0.5 * (hy - ly) + mx; b.ez = 0.5 * (hz - lz) + mx;
    return b;
}

// Per-axis distance of a coordinate from a box centre, at the nearest periodic image
// (a zero period, as an open set passes to the periodic form, folds nothing).
template<bool Periodic>
__device__ __forceinline__ double axis_dist(double x, double c, double L)
{
    double d = fabs(x - c);
    if (Periodic && L > 0.0) d = fmin(d, L - d);
    return d;
}

// Gather filter: inside the group's box of search spheres.
template<bool Periodic>
__device__ __forceinline__ bool in_gather_box(const double4& p, const GroupBox& b, double lx, double ly, double lz)
{
    return axis_dist<Periodic>(p.x, b.cx, lx) <= b.ex && axis_dist<Periodic>(p.y, b.cy, ly) <= b.ey &&
           axis_dist<Periodic>(p.z, b.cz, lz) <= b.ez;
}

// A rounded box: the points within r of the box (c, e) -- the members' own bounding box
// and their largest support.  Every pair a member accepts has its j inside (the distance
// from j to the box is at most the distance to that member), and the region leaves out the
// cube's corners and edges: about a fifth of the cube for a 32-particle group of a uniform
// lattice, and, for a single particle (a box of zero size), all but its sphere.  r < 0: none.
struct RoundBox
{
    double cx, cy, cz, ex, ey, ez, r;
};

template<bool Periodic>
__device__ __forceinline__ bool in_round_box(const double4& p, const RoundBox& b, double lx, double ly, double lz)
{
    const double gx = fmax(axis_dist<Periodic>(p.x, b.cx, lx) - b.ex, 0.0);
    const double gy = fmax(axis_dist<Periodic>(p.y, b.cy, ly) - b.ey, 0.0);
    const double gz = fmax(axis_dist<Periodic>(p.z, b.cz, lz) - b.ez, 0.0);
    return gx * gx + gy * gy + gz * gz <= b.r * b.r;
}

// Symmetric filter: within R*max(hmax_group, h_j) of the box of the group's positions.
template<bool Periodic>
__device__ __forceinline__ bool in_sym_box(const double4& p, const GroupBox& b, double rg, double lx, double ly,
                                           double lz)
{
    const double gx = axis_dist<Periodic>(p.x, b.cx, lx) - b.ex;
    const double gy = axis_dist<Periodic>(p.y, b.cy, ly) - b.ey;
    const double gz = axis_dist<Periodic>(p.z, b.cz, lz) - b.ez;
    const double dx = gx > 0.0 ? gx : 0.0, dy = gy > 0.0 ? gy : 0.0, dz = gz > 0.0 ? gz : 0.0;
    const double r = fmax(rg, kRadKernel * p.w) * (1.0 + 1e-9);
    return dx * dx + dy * dy + dz * dz <= r * r;
}

__device__ __forceinline__ uint32_t warp_incl_scan_u32(uint32_t v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// The particle range of a j-leaf: layout[leaf] .. layout[leaf + 1] for a single set,
// or a table of (begin, end) pairs for a forest.
struct LayoutRanges
{
    const uint32_t* __restrict__ layout;
    __device__ __forceinline__ uint2 operator()(int leaf) const { return make_uint2(layout[leaf], layout[leaf + 1]); }
};

struct TableRanges
{
    const uint2* __restrict__ range;
    __device__ __forceinline__ uint2 operator()(int leaf) const { return range[leaf]; }
};

// Signed offset of x from c at the nearest periodic image (L > 0), or plain (L == 0).
__device__ __forceinline__ double image_offset(double x, double c, double L)
{
    double d = x - c;
    if (L > 0.0)
    {
        if (d > 0.5 * L) d -= L;
        else if (d < -0.5 * L) d += L;
    }
    return d;
}

// The warp's candidate ring: j particles that pass the group filter are compacted into
// it, in order, and handed to batch(ring, ringf, ringIdx, head, count) in runs of up to 32
// on every lane.  The ring keeps what the caller asks for: the FP64 xyzh (Dbl), an FP32
// copy relative to the group box centre at the nearest periodic image when lx, ly, lz > 0
// (Float), and the particle index (Index).
template<bool Dbl, bool Float, bool Index, bool Staged = false>
struct CandidateRing
{
    double4* ring;
    float4* ringf;
    int* ringIdx;
    double cx, cy, cz, lx, ly, lz;
    StageRef stage;
    int head = 0, cnt = 0;

    template<class Batch>
    __device__ __forceinline__ void drain(int count, Batch& batch)
    {
        batch(ring, ringf, ringIdx, head, count);
        head = (head + count) & (kRing - 1);
        cnt -= count;
        __syncwarp();
    }

    // Stream the particle ranges held one per lane (s0, len; lanes >= nb hold none), in
    // lane order.  A warp prefix sum over the lengths flattens them, so every load batch is
    // 32 consecutive stream positions (each lane finds its particle by a 5-step binary
    // search over the prefix sums), and the next batch's loads are issued before the
    // current batch is filtered.  filter(pj) is evaluated by the loading lane only.
    template<class Filter, class Batch>
    __device__ __forceinline__ void feed(uint32_t s0, uint32_t len, int nb, const double4* __restrict__ xyzh,
                                         Filter& filter, Batch& batch)
    {
        if constexpr (Staged)
            if (stage.ws->broken == 0u)
            {
                feed_staged(s0, len, nb, xyzh, filter, batch);
                return;
            }
        const int lane = threadIdx.x & 31;
        const uint32_t lt = (1u << lane) - 1u;
        const uint32_t incl = warp_incl_scan_u32(len);
        const uint32_t excl = incl - len;
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        // particle index of stream position p (p < total)
        auto locate = [&](uint32_t p) -> uint32_t {
            int t = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1)
            {
                const uint32_t e = __shfl_sync(0xffffffffu, excl, (t + step) & 31);
                if (t + step < nb && e <= p) t += step;
            }
            return __shfl_sync(0xffffffffu, s0, t) + (p - __shfl_sync(0xffffffffu, excl, t));
        };
        uint32_t j = 0;
        double4 pj = make_double4(0, 0, 0, 0);
        if (total > 0)
        {
            j = locate(lane);
            if (uint32_t(lane) < total) pj = ldg4(xyzh + j);
        }
        for (uint32_t p0 = 0; p0 < total; p0 += 32)
        {
            const bool valid = p0 + lane < total;
            uint32_t jn = 0;
            double4 pn = make_double4(0, 0, 0, 0);
            if (p0 + 32 < total)
            {
                jn = locate(p0 + 32 + lane);
                if (p0 + 32 + lane < total) pn = ldg4(xyzh + jn);
            }
            const bool pass = valid && filter(pj);
            const uint32_t m = __ballot_sync(0xffffffffu, pass);
            if (pass)
            {
                const int slot = (head + cnt + __popc(m & lt)) & (kRing - 1);
                if constexpr (Dbl) ring[slot] = pj;
                if constexpr (Float)
                    ringf[slot] = make_float4(float(image_offset(pj.x, cx, lx)), float(image_offset(pj.y, cy, ly)),
                                              float(image_offset(pj.z, cz, lz)), float(pj.w));
                if constexpr (Index) ringIdx[slot] = int(j);
            }
            cnt += __popc(m);
            __syncwarp();
            if (cnt >= 32) drain(32, batch);
            j = jn;
            pj = pn;
        }
    }

    // Admit one loaded stream position (pj, particle index j) through the filter into the
    // ring, in order, and hand full batches of 32 to batch.
    template<class Filter, class Batch>
    __device__ __forceinline__ void admit(bool valid, const double4& pj, uint32_t j, Filter& filter, Batch& batch)
    {
        const int lane = threadIdx.x & 31;
        const uint32_t lt = (1u << lane) - 1u;
        const bool pass = valid && filter(pj);
        const uint32_t m = __ballot_sync(0xffffffffu, pass);
        if (pass)
        {
            const int slot = (head + cnt + __popc(m & lt)) & (kRing - 1);
            if constexpr (Dbl) ring[slot] = pj;
            if constexpr (Float)
                ringf[slot] = make_float4(float(image_offset(pj.x, cx, lx)), float(image_offset(pj.y, cy, ly)),
                                          float(image_offset(pj.z, cz, lz)), float(pj.w));
            if constexpr (Index) ringIdx[slot] = int(j);
        }
        cnt += __popc(m);
        __syncwarp();
        if (cnt >= 32) drain(32, batch);
    }

    // feed() with the stream staged by bulk copies: chunk c (stream positions 32c ..
    // 32c + 31) is copied into stage buffer c % kStages as one cp.async.bulk per run of
    // consecutive particles (a run starts where the particle index does not follow its
    // predecessor's; Hilbert-ordered leaves make runs of whole leaves and more), issued by
    // the run's first lane and completing on the buffer's mbarrier.  While chunk c is
    // filtered, chunk c + 1 is in flight.  A wait that gives up raises kErrStageWait,
    // waits (bounded) for the copies still in flight, marks the stage broken and returns;
    // the host then reports the error.
    template<class Filter, class Batch>
    __device__ __forceinline__ void feed_staged(uint32_t s0, uint32_t len, int nb, const double4* __restrict__ xyzh,
                                                Filter& filter, Batch& batch)
    {
        const int lane = threadIdx.x & 31;
        WarpStage& S = *stage.ws;
        const uint32_t incl = warp_incl_scan_u32(len);
        const uint32_t excl = incl - len;
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        auto locate = [&](uint32_t p) -> uint32_t {
            int t = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1)
            {
                const uint32_t e = __shfl_sync(0xffffffffu, excl, (t + step) & 31);
                if (t + step < nb && e <= p) t += step;
            }
            return __shfl_sync(0xffffffffu, s0, t) + (p - __shfl_sync(0xffffffffu, excl, t));
        };
        const uint32_t nChunks = (total + 31u) >> 5;
        uint32_t phase = S.phase;
        auto issue = [&](uint32_t c) {
            const int b = int(c % kStages);
            const uint32_t p = (c << 5) + uint32_t(lane);
            const bool valid = p < total;
            const uint32_t j = locate(p);
            const uint32_t jp = __shfl_up_sync(0xffffffffu, j, 1);
            const bool start = valid && (lane == 0 || j != jp + 1u);
            const uint32_t starts = __ballot_sync(0xffffffffu, start);
            const int count = int(min(32u, total - (c << 5)));
            if (lane == 0) mbar_arrive_expect_tx(&S.bar[b], uint32_t(count) * 32u);
            __syncwarp();
            if (start)
            {
                const uint32_t after = starts & ~((2u << lane) - 1u);
                const int end = after ? (__ffs(after) - 1) : count;
                bulk_g2s(&S.buf[b][lane], xyzh + j, uint32_t(end - lane) * 32u, &S.bar[b]);
            }
        };
        for (uint32_t c = 0; c < nChunks && c < uint32_t(kStages); ++c) issue(c);
        for (uint32_t c = 0; c < nChunks; ++c)
        {
            const int b = int(c % kStages);
            // lane 0 waits under the limit; once it has seen the phase complete, the other
            // lanes' waits (each lane's own acquire of the copied data) return at once
            bool got = lane == 0 ? mbar_wait_bounded(&S.bar[b], (phase >> b) & 1u, stage.limitNs) : true;
            got = __shfl_sync(0xffffffffu, got, 0);
            if (got && lane != 0) mbar_wait_bounded(&S.bar[b], (phase >> b) & 1u, stage.limitNs);
            if (!got)
            {
                // give up: the copies still in flight (this chunk's and those after it) must
                // land before the warp leaves the buffers
                if (lane == 0) atomicOr(stage.err, int(kErrStageWait));
                const uint32_t last = min(nChunks, c + uint32_t(kStages));
                if (lane == 0)
                {
                    for (uint32_t d = c; d < last; ++d)
                    {
                        const int bd = int(d % kStages);
                        mbar_wait_bounded(&S.bar[bd], (phase >> bd) & 1u, stage.limitNs);
                    }
                    S.broken = 1u;
                }
                __syncwarp();
                return;
            }
            phase ^= 1u << b;
            const uint32_t p = (c << 5) + uint32_t(lane);
            const bool valid = p < total;
            double4 pj = make_double4(0, 0, 0, 0);
            if (valid) pj = S.buf[b][lane];
            const uint32_t j = Index ? locate(p) : 0u;
            fence_proxy_async_smem();   // the reads above before the next copy into buffer b
            __syncwarp();
            if (c + uint32_t(kStages) < nChunks) issue(c + uint32_t(kStages));
            admit(valid, pj, j, filter, batch);
        }
        if (lane == 0) S.phase = phase;
        __syncwarp();
    }

    template<class Batch>
    __device__ __forceinline__ void finish(Batch& batch)
    {
        if (cnt > 0) drain(cnt, batch);
    }
};

// Stream the j particles of one i-leaf list (entries jb .. jb + nj of jlist, in order)
// through the group filter into the ring, 32 list entries at a time.
template<bool Dbl, bool Float, bool Index, bool Staged = false, class Ranges, class Filter, class Batch>
__device__ __forceinline__ void stream_ranges(double4* ring, float4* ringf, int* ringIdx, double cx, double cy,
                                              double cz, double lx, double ly, double lz, uint32_t jb, uint32_t nj,
                                              const int* __restrict__ jlist, Ranges ranges,
                                              const double4* __restrict__ xyzh, Filter filter, Batch batch,
                                              StageRef stage = StageRef{nullptr, nullptr, 0})
{
    const int lane = threadIdx.x & 31;
    CandidateRing<Dbl, Float, Index, Staged> cr{ring, ringf, ringIdx, cx, cy, cz, lx, ly, lz, stage};
    for (uint32_t lb = 0; lb < nj; lb += 32)
    {
        const int nb = int(min(32u, nj - lb));
        uint32_t s0 = 0, len = 0;
        if (lane < nb)
        {
            const uint2 r = ranges(jlist[jb + lb + lane]);
            s0 = r.x;
            len = r.y - r.x;
        }
        cr.feed(s0, len, nb, xyzh, filter, batch);
    }
    cr.finish(batch);
}

// The pre-order node arrays of a tree (or of one set's range [n0, n1) of a forest) for
// stream_walk.
struct PreorderTree
{
    const double4* __restrict__ center;
    const double4* __restrict__ half;
    const int* __restrict__ skip;
    const int* __restrict__ leaf;
    int n0, n1;
    const int* n1p = nullptr;   // when given, the end node n1 is read here (a captured graph)
};

// Stream the j particles of every leaf whose cell overlaps the box (c, e) -- and the
// region (rc, re), when re.x >= 0, and the rounded box *rbp, when given -- through the
// group filter into the ring, found by a stackless pre-order scan of the tree 32 nodes at
// a time (the scan of list_walk_kernel): leaves come out in ascending order, so the
// stream is in ascending j as a list's is.  Used for groups whose leaf list is far longer
// than their own search region needs.  A group's cube can hold far more than its rounded
// box (a large h near the edge of a centrally concentrated set: the cube of a single
// particle reaches the dense core, its sphere does not), so cells are tested on both.
template<bool Dbl, bool Float, bool Index, bool Periodic, bool Staged = false, class Ranges, class Filter,
         class Batch>
__device__ __forceinline__ void stream_walk(double4* ring, float4* ringf, int* ringIdx, double cx, double cy,
                                            double cz, double sx, double sy, double sz, const PreorderTree& t,
                                            double3 c, double3 e, double3 rc, double3 re, double lx, double ly,
                                            double lz, Ranges ranges, const double4* __restrict__ xyzh,
                                            Filter filter, Batch batch, StageRef stage = StageRef{nullptr, nullptr, 0},
                                            const RoundBox* rbp = nullptr)
{
    const int lane = threadIdx.x & 31;
    CandidateRing<Dbl, Float, Index, Staged> cr{ring, ringf, ringIdx, cx, cy, cz, sx, sy, sz, stage};
    auto fold = [&](double d, double L) { return (Periodic && L > 0.0) ? fmin(d, L - d) : d; };
    const int n1 = t.n1p != nullptr ? *t.n1p : t.n1;
    int p = t.n0;
    while (p < n1)
    {
        const int idx = p + lane;
        const bool valid = idx < n1;
        bool accept = false;
        int skip = 1, pl = -1;
        if (valid)
        {
            const double4 nc = t.center[idx];
            const double4 nh = t.half[idx];
            accept = fold(fabs(c.x - nc.x), lx) <= e.x + nh.x && fold(fabs(c.y - nc.y), ly) <= e.y + nh.y &&
                     fold(fabs(c.z - nc.z), lz) <= e.z + nh.z;
            if (re.x >= 0.0)
                accept = accept && fold(fabs(rc.x - nc.x), lx) <= re.x + nh.x &&
                         fold(fabs(rc.y - nc.y), ly) <= re.y + nh.y && fold(fabs(rc.z - nc.z), lz) <= re.z + nh.z;
            if (rbp != nullptr)
            {
                // gap between the rounded box's core and the cell, per axis then squared
                const RoundBox rb = *rbp;
                const double gx = fmax(fold(fabs(rb.cx - nc.x), lx) - nh.x - rb.ex, 0.0);
                const double gy = fmax(fold(fabs(rb.cy - nc.y), ly) - nh.y - rb.ey, 0.0);
                const double gz = fmax(fold(fabs(rb.cz - nc.z), lz) - nh.z - rb.ez, 0.0);
                accept = accept && gx * gx + gy * gy + gz * gz <= rb.r * rb.r;
            }
            skip = t.skip[idx];
            pl = t.leaf[idx];
        }
        const uint32_t validMask = __ballot_sync(0xffffffffu, valid);
        const uint32_t rejMask = __ballot_sync(0xffffffffu, valid && !accept);
        // the reached, accepted leaves of this window, in lane (pre-) order
        uint32_t emit = 0;
        int pos = 0, next = p + 32;
        for (;;)
        {
            const uint32_t fromPos = (pos >= 32) ? 0u : (0xffffffffu << pos);
            const uint32_t rej = rejMask & fromPos;
            const int r = rej ? (__ffs(rej) - 1) : 32;
            const uint32_t runMask = validMask & fromPos & ((r >= 32) ? 0xffffffffu : ((1u << r) - 1u));
            emit |= runMask;
            if (r >= 32) { next = p + 32; break; }
            int rskip = __shfl_sync(0xffffffffu, skip, r);
            if (rskip < 1) rskip = 1;   // a subtree holds its root: the scan always advances
            const int target = p + r + rskip;
            if (target >= p + 32 || target >= n1) { next = target; break; }
            pos = target - p;
        }
        emit &= __ballot_sync(0xffffffffu, pl >= 0);
        if (emit)
        {
            // compact the emitted leaves onto the low lanes, keeping their order
            const bool mineLeaf = (emit >> lane) & 1u;
            const int nb = __popc(emit);
            uint2 r = make_uint2(0, 0);
            if (mineLeaf) r = ranges(pl);
            // lane k takes the k-th emitted leaf's range
            const unsigned src = __fns(emit, 0, lane + 1);
            const int sl = src < 32u ? int(src) : 0;
            const uint32_t rx = __shfl_sync(0xffffffffu, r.x, sl);
            const uint32_t ry = __shfl_sync(0xffffffffu, r.y, sl);
            const uint32_t s0 = lane < nb ? rx : 0u, len = lane < nb ? ry - rx : 0u;
            cr.feed(s0, len, nb, xyzh, filter, batch);
        }
        p = next;
    }
    cr.finish(batch);
}

// Where a group's candidates come from: its leaf's j-leaf list (entries jb .. jb + nj of
// jlist), or, when walk is set, a pre-order scan of the tree for the leaves overlapping
// the group's own box, within the leaf list's region (rc, re).
template<class Ranges>
struct GroupSource
{
    const int* __restrict__ jlist;
    uint32_t jb, nj;
    Ranges ranges;
    const double4* __restrict__ xyzh;
    bool walk;
    PreorderTree tree;
    double3 rc, re;
    StageRef stage;   // the warp's bulk-copy stage, or none (direct loads)

    // rbp (when given): the group's rounded box, for the tree scan's cells
    template<bool Dbl, bool Float, bool Index, bool Periodic, bool Staged = false, class Filter, class Batch>
    __device__ __forceinline__ void stream(double4* ring, float4* ringf, int* ringIdx, const GroupBox& bx, double sx,
                                           double sy, double sz, double lx, double ly, double lz, Filter filter,
                                           Batch batch, const RoundBox* rbp = nullptr) const
    {
        if (walk)
            stream_walk<Dbl, Float, Index, Periodic, Staged>(ring, ringf, ringIdx, bx.cx, bx.cy, bx.cz, sx, sy, sz, tree,
                                                     make_double3(bx.cx, bx.cy, bx.cz),
                                                     make_double3(bx.ex, bx.ey, bx.ez), rc, re, lx, ly, lz, ranges,
                                                     xyzh, filter, batch, stage, rbp);
        else
            stream_ranges<Dbl, Float, Index, Staged>(ring, ringf, ringIdx, bx.cx, bx.cy, bx.cz, sx, sy, sz, jb, nj,
                                                     jlist, ranges, xyzh, filter, batch, stage);
    }
};

template<class Ranges>
__device__ __forceinline__ GroupSource<Ranges> list_source(const int* jlist, uint32_t jb, uint32_t nj, Ranges ranges,
                                                           const double4* xyzh)
{
    GroupSource<Ranges> g{jlist, jb, nj, ranges, xyzh, false, PreorderTree{nullptr, nullptr, nullptr, nullptr, 0, 0},
                          make_double3(0, 0, 0), make_double3(-1, -1, -1), StageRef{nullptr, nullptr, 0}};
    return g;
}

// stream_ranges over a single set's leaves, FP32 copies relative to the box centre
// without periodic shift (the pair tests fold the images themselves).
template<bool Float = true, bool Index = true, class Filter, class Batch>
__device__ __forceinline__ void stream_pairs(double4* ring, float4* ringf, int* ringIdx, double cx, double cy,
                                             double cz, uint32_t jb, uint32_t nj, const int* __restrict__ jlist,
                                             const uint32_t* __restrict__ layout,
                                             const double4* __restrict__ xyzh, Filter filter, Batch batch)
{
    stream_ranges<true, Float, Index>(ring, ringf, ringIdx, cx, cy, cz, 0.0, 0.0, 0.0, jb, nj, jlist,
                                      LayoutRanges{layout}, xyzh, filter, batch);
}

// Two passes over one batch of up to 32 ring entries, for a lane's own particle:
//   A  test(pf) on the float copy, branch-free, collected into a 32-bit mask.  It is a
//      CONSERVATIVE prefilter: it may pass a pair the exact test rejects, never the
//      reverse (see fp32_margin);
//   B  for the set bits in ascending order (all lanes in lockstep until every lane's
//      mask is empty), accept(pj, pf, j) applies the exact test and evaluates the pair.
// The order in which a lane accepts its pairs is the ring order, i.e. ascending j.
template<class Test, class Accept>
__device__ __forceinline__ void two_pass(const double4* ring, const float4* ringf, const int* ringIdx, int head,
                                         int count, bool mine, Test test, Accept accept)
{
    uint32_t acc = 0;
#pragma unroll 8
    for (int k = 0; k < count; ++k)
        acc |= (test(ringf[(head + k) & (kRing - 1)]) ? 1u : 0u) << k;
    if (!mine) acc = 0;
    while (__any_sync(0xffffffffu, acc != 0))
    {
        if (acc)
        {
            const int k = __ffs(acc) - 1;
            acc &= acc - 1;
            const int s = (head + k) & (kRing - 1);
            accept(ring[s], ringf[s], ringIdx[s]);
        }
    }
}

// Absolute error bound of a float-relative-coordinate distance for a group.  Relative
// coordinates are at most A = the box half extent (plus the period when periodic).  Per
// axis, the two conversions, the subtraction and the periodic fold each round by at most
// 2A*2^-24, so |d_float - |dx|| <= 6A*2^-24 and the 3-vector error is below
// sqrt(3)*6A*2^-24 < 11A*2^-24; 16A*2^-24 covers it with room.  Relative rounding of
// the squares and sums is covered by the caller's (1 + 1e-6) or (1 + 1e-5) factor.
__device__ __forceinline__ double fp32_margin(const GroupBox& b, double period)
{
    const double A = fmax(b.ex, fmax(b.ey, b.ez)) + period;
    return 16.0 * A * 5.9604644775390625e-8;
}

// Bound on the FP32 squared distance r2_f of a pair whose exact distance is below B, for
// a group whose float offsets carry the absolute error eps of fp32_margin.  Per axis the
// float separation of offsets a (|a| <= A) and b errs by at most 2^-24 (|a| + |b| + |d|)
// <= 2^-23 (A + |d|) (open: |b| <= |a| + |d|; periodic: the fold's terms are absolute and
// inside eps), so over three axes r_f <= r (1 + 2^-23) + eps and r2_f <= r_f^2 (1 + 3 2^-24):
// r < B implies r2_f < (B (1 + 1e-6) + eps)^2 (1 + 1e-6).  A candidate far outside the
// group box (a scatter neighbour of large h) is covered by the relative term.
__device__ __forceinline__ float fp32_bound2(double B, double eps)
{
    const double t = B * (1.0 + 1e-6) + eps;
    return float(t * t * (1.0 + 1e-6));
}

// Per-axis float distance, at the nearest periodic image when periodic.
template<bool Periodic>
__device__ __forceinline__ float axis_df(float a, float b, float L)
{
    float d = fabsf(a - b);
    if (Periodic) d = fminf(d, L - d);
    return d;
}

template<bool Periodic>
__device__ __forceinline__ float r2_f32(float xi, float yi, float zi, const float4& pf, float Lx, float Ly, float Lz)
{
    const float dx = axis_df<Periodic>(xi, pf.x, Lx);
    const float dy = axis_df<Periodic>(yi, pf.y, Ly);
    const float dz = axis_df<Periodic>(zi, pf.z, Lz);
    return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
}

// Near-equal split of a leaf window's active slots into warp groups: group g of G takes
// active ranks [g*nAct/G, (g+1)*nAct/G).  Returns the lane's slot in the 64-slot window
// (or -1) via kth set bit of (lo | hi << 32).
__device__ __forceinline__ int group_slot(uint32_t lo, uint32_t hi, int nAct, int g, int G, int lane)
{
    const int k0 = g * nAct / G, k1 = (g + 1) * nAct / G;
    int k = k0 + lane;
    if (k >= k1) return -1;
    const int nlo = __popc(lo);
    if (k < nlo) return int(__fns(lo, 0, k + 1));
    k -= nlo;
    return 32 + int(__fns(hi, 0, k + 1));
}

// Compensated (Kahan) FP32 accumulation; the exact sum is s - c, formed in FP64.
struct KahanF
{
    float s = 0.0f, c = 0.0f;
    __device__ __forceinline__ void add(float x)
    {
        const float y = x - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double value() const { return double(s) - double(c); }
};

// The SPH kernel in FP32 (same polynomials as sph_kernel).
__device__ __forceinline__ void sph_kernel_f(float q2, float q, float& w, float& dw)
{
    if constexpr (kQuintic)
    {
        if (q < 1.0f)
        {
            const float q4 = q2 * q2;
            w  = fmaf(-10.0f * q4, q, fmaf(30.0f, q4, fmaf(-60.0f, q2, 66.0f)));
            dw = q * fmaf(-50.0f * q2, q, fmaf(120.0f, q2, -120.0f));
        }
        else if (q < 2.0f)
        {
            const float a = q - 3.0f, b = q - 2.0f;
            const float a2 = a * a, b2 = b * b;
            w  = fmaf(6.0f, b2 * b2 * b, -(a2 * a2 * a));
            dw = fmaf(30.0f, b2 * b2, -5.0f * (a2 * a2));
        }
        else if (q < 3.0f)
        {
            const float a = q - 3.0f, a2 = a * a;
            w  = -(a2 * a2 * a);
            dw = -5.0f * (a2 * a2);
        }
        else { w = 0.0f; dw = 0.0f; }
    }
    else
    {
        (void)q2;
        const float a = fmaxf(2.0f - q, 0.0f), b = fmaxf(1.0f - q, 0.0f);
        const float a2 = a * a, b2 = b * b;
        w  = 0.25f * fmaf(-4.0f * b2, b, a2 * a);
        dw = 0.25f * fmaf(12.0f, b2, -3.0f * a2);
    }
}

} // namespace cosmo
