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
 * Row layout: kNbl entries per particle (row i at nbl + i * kNbl, 16-byte aligned); a
 * count above kNbl marks a row that overflowed, whose particle keeps the group path.
 */
#pragma once

#include "pairstream.cuh"

namespace cosmo {

constexpr int kNbl = kQuintic ? 256 : 128;

// Per-warp shared scratch of rows_group: the double ring, its indices, the group's data.
constexpr int kRowsScratch = kRing * 32 + kRing * 4 + 32 * 32;

// Rows of one group.  Lanes [0, ng) own the group's particles, whose per-particle test data
// gi (a double4: position and one test value) the caller passes; test(gi, pj) is the exact
// acceptance of the pair.  row is the lane's own row (nullptr if not mine); rowLen
// receives its length (kNbl + 1 when it overflowed).
template<class Ranges, class Filter, class Test>
__device__ __forceinline__ void rows_group(unsigned char* scr, bool mine, int ng, const double4& gi, const GroupBox& bx,
                                           uint32_t jb, uint32_t nj, const int* __restrict__ jlist, Ranges ranges,
                                           const double4* __restrict__ xyzh, Filter filter, Test test, int* row,
                                           int& rowLen)
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
                if (len < kNbl) row[len] = ri[(head + b) & (kRing - 1)];
                ++len;
            }
        });
    rowLen = len > kNbl ? kNbl + 1 : len;
}

// Whether particle i's row is usable (written and not overflowed).
__device__ __forceinline__ bool row_ok(const int* __restrict__ nblCount, uint32_t i)
{
    return unsigned(nblCount[i]) <= unsigned(kNbl);
}

} // namespace cosmo
