/*
 * rows.cuh -- neighbour rows: each particle's accepted j, in ascending order, written once
 * by a group pass so that the heavy pair passes run with one lane per particle.
 *
 * The group pass streams a leaf's list through the group filter into the warp's ring and
 * tests each batch with j on the lanes (for each group particle in turn, every lane tests
 * its candidate); the ballot of a group particle's tests is its lane's mask over the
 * batch, and the owner lane appends the masked j, lowest lane first -- ascending j.  A pass
 * that then walks a row applies the same exact test to the same candidates in the same
 * order as a walk of the whole list would, so its sums are the same bit for bit.
 *
 * An entry is j (the symmetric rows of the gradient and force passes), or r^2 of the pair
 * (the Newton rows: positions do not move during a density solve, so the later Newton
 * iterations need only r^2 and h_i, and read no j data at all).  The Newton rows are flat
 * (kNbl consecutive entries per particle, FP64, or FP32 in the mixed form): their reader
 * streams its own row 16-32 bytes at a time, so the sectors it touches hold only its own
 * entries whichever particles share its warp.
 *
 * Row layout: kNbl entries per particle, interleaved over blocks of 32 particles -- entry
 * k of particle i at nbl[(i / 32) * 32 kNbl + 32 k + i % 32] -- so that the lanes of a warp
 * over 32 consecutive particles read entry k of all their rows from one 128-byte line.  A
 * count above kNbl marks a row that overflowed, whose particle keeps the group path.
 */
#pragma once

#include "pairstream.cuh"

namespace cosmo {

constexpr int kNbl = kQuintic ? 256 : 128;
constexpr int kRowStride = 32;   // distance between consecutive entries of one row

// Entries the row buffer of n particles holds.
inline size_t row_buffer_entries(size_t n) { return ((n + 31) / 32) * size_t(32) * kNbl; }

// Entry 0 of particle i's row; entry k is at [k * kRowStride].
template<class T>
__device__ __forceinline__ T* row_of(T* nbl, uint32_t i)
{
    return nbl + (size_t(i >> 5) * kNbl << 5) + (i & 31u);
}

// Per-warp shared scratch of rows_group: the double ring, its indices, the group's data.
constexpr int kRowsScratch = kRing * 32 + kRing * 4 + 32 * 32;

// Rows of one group.  Lanes [0, ng) own the group's particles, whose per-particle test data
// gi (a double4: position and one test value) the caller passes; test(gi, pj) is the exact
// acceptance of the pair, and value(pj, j) the entry the owner writes for an accepted j (j
// itself, or a pair quantity it recomputes from pj).  row is the lane's own row (row_of
// with Stride kRowStride, or row_flat with Stride 1; nullptr if not mine); rowLen receives
// its length (kNbl + 1 when it overflowed).
template<int Stride, class T, class Ranges, class Filter, class Test, class Value>
__device__ __forceinline__ void rows_group(unsigned char* scr, bool mine, int ng, const double4& gi, const GroupBox& bx,
                                           uint32_t jb, uint32_t nj, const int* __restrict__ jlist, Ranges ranges,
                                           const double4* __restrict__ xyzh, Filter filter, Test test, Value value,
                                           T* row, int& rowLen)
{
    const int lane = threadIdx.x & 31;
    double4* ring = reinterpret_cast<double4*>(scr);
    int* ringIdx = reinterpret_cast<int*>(ring + kRing);
    double4* grp = reinterpret_cast<double4*>(ringIdx + kRing);
    if (mine) grp[lane] = gi;
    __syncwarp();
    int len = 0;
    stream_ranges<true, false, true>(
        ring, nullptr, ringIdx, bx.cx, bx.cy, bx.cz, 0.0, 0.0, 0.0, jb, nj, jlist, ranges, xyzh, filter,
        [&](const double4* rg, const float4*, const int* ri, int head, int count) {
            const double4 pj = rg[(head + (lane < count ? lane : 0)) & (kRing - 1)];
            uint32_t myMask = 0;
            for (int i0 = 0; i0 < ng; i0 += 4)
            {
                bool a[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) a[u] = lane < count && i0 + u < ng && test(grp[min(i0 + u, 31)], pj);
#pragma unroll
                for (int u = 0; u < 4; ++u)
                {
                    const uint32_t m = __ballot_sync(0xffffffffu, a[u]);
                    if (lane == i0 + u) myMask = m;
                }
            }
            while (myMask)
            {
                const int b = __ffs(myMask) - 1;
                myMask &= myMask - 1;
                const int sl = (head + b) & (kRing - 1);
                if (len < kNbl) row[size_t(len) * Stride] = value(rg[sl], ri[sl]);
                ++len;
            }
        });
    rowLen = len > kNbl ? kNbl + 1 : len;
}

// Entry 0 of particle i's row in the flat layout (kNbl consecutive entries per particle).
template<class T>
__device__ __forceinline__ T* row_flat(T* nbl, uint32_t i)
{
    return nbl + size_t(i) * kNbl;
}

// f(r2) for the cnt entries of a flat row of doubles, in order, 32 bytes per load (the
// rows are 32-byte aligned and kNbl is a multiple of 4, so the last load stays in the row).
template<class F>
__device__ __forceinline__ void for_flat_row(const double* __restrict__ row, int cnt, F&& f)
{
    const double4* r4 = reinterpret_cast<const double4*>(row);
    int k = 0;
    for (; k + 4 <= cnt; k += 4)
    {
        const double4 v = ldg4(r4 + (k >> 2));
        f(v.x); f(v.y); f(v.z); f(v.w);
    }
    if (k < cnt)
    {
        const double4 v = ldg4(r4 + (k >> 2));
        f(v.x);
        if (k + 1 < cnt) f(v.y);
        if (k + 2 < cnt) f(v.z);
    }
}

// The same over a flat row of floats (the mixed form's r^2 rows), 16 bytes per load.
template<class F>
__device__ __forceinline__ void for_flat_row(const float* __restrict__ row, int cnt, F&& f)
{
    const float4* r4 = reinterpret_cast<const float4*>(row);
    int k = 0;
    for (; k + 4 <= cnt; k += 4)
    {
        const float4 v = __ldg(r4 + (k >> 2));
        f(v.x); f(v.y); f(v.z); f(v.w);
    }
    if (k < cnt)
    {
        const float4 v = __ldg(r4 + (k >> 2));
        f(v.x);
        if (k + 1 < cnt) f(v.y);
        if (k + 2 < cnt) f(v.z);
    }
}

// f(entry) for the cnt entries of a row (row_of), in order, four loads ahead of their use.
template<class T, class F>
__device__ __forceinline__ void for_row(const T* __restrict__ row, int cnt, F&& f)
{
    int k = 0;
    for (; k + 4 <= cnt; k += 4)
    {
        const T a = __ldg(row + size_t(k) * kRowStride), b = __ldg(row + size_t(k + 1) * kRowStride);
        const T c = __ldg(row + size_t(k + 2) * kRowStride), d = __ldg(row + size_t(k + 3) * kRowStride);
        f(a); f(b); f(c); f(d);
    }
    for (; k < cnt; ++k) f(__ldg(row + size_t(k) * kRowStride));
}

// Whether particle i's row is usable (written and not overflowed).
__device__ __forceinline__ bool row_ok(const int* __restrict__ nblCount, uint32_t i)
{
    return unsigned(nblCount[i]) <= unsigned(kNbl);
}

} // namespace cosmo
